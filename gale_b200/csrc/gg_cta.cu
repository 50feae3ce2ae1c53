// gg_cta.cu -- the batched Uzawa solver: one CTA solves one whole problem, and one launch
// solves the whole batch (the uneven sweep of many small independent problems).
//
// The per-handle path drives each problem from the host: every inner solve is at least one
// cooperative launch followed by a host synchronisation, every Uzawa step a few more, so a
// 64² sinker spends most of its time waiting for the host.  Here a persistent kernel pulls
// problem indices from a device work queue (largest problems first); the CTA that takes a
// problem runs all of it on one SM with block barriers only:
//   multigrid set-up  coarse moments (exact re-expansion of the children's), coarse BC
//                     masks, Jacobi diagonals, λ_max by 12 power steps per level, the
//                     coarsest operator assembled into shared memory and inverted there by
//                     Gauss–Jordan (FP32);
//   Uzawa             _Stokes_SLE_UzawaSolver_Solve (Stokes_SLE_UzawaSolver.cxx:393-938)
//                     step for step, FP64, Ĝ-preconditioned, as gg_solve.cu:uzawa_solve;
//   inner solves      FP64 defect correction around FP32 flexible-CG sweeps preconditioned
//                     by a Chebyshev–Jacobi V-cycle, the stopping rules of inner_solve;
//   element applies   the matrix-free kernel of gg_ops.cuh over the element parity classes
//                     with a block barrier between classes: no two threads add into the same
//                     node at once, and every node sums its element terms in class order, so
//                     a problem solved here gives the same bits on every run.
// Vectors live in global memory (L2-resident for these sizes); inside the launch they are
// read with L1-cached loads, coherent within the CTA across its block barriers.
#include <math.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"
#include "gg_ops.cuh"

namespace gg {

MeshK make_mesh(const gg_mesh_desc& d);

namespace {

// threads per CTA: 512 in 2D (≤ 128 registers, 16 warps per SM), 256 in 3D, where the FP64
// element apply needs ~220 registers
template <int DIM>
constexpr int cta_threads() { return DIM == 2 ? 512 : 256; }
constexpr int kCtaMaxLevels = 8;
constexpr int kCtaDenseMax = 200;  // dofs of a coarsest level inverted in shared memory
constexpr int kCtaMinCoarse = 4;   // coarsen while every axis is even and ≥ 4 elements
constexpr int kCtaPowerSteps = 12;
constexpr int kCtaCoarseChebDegree = 8;  // coarsest level without the dense inverse

struct CtaLevel {
    MeshK mk;
    double* mom64;  // level 0: the handle's FP64 moments; coarse levels: written here
    float* mom32;
    uint8_t* bc;
    float* invd;
    float *x, *b, *r, *d, *t;
};

struct CtaProblem {
    int nlevels;   // levels 0 .. nlevels−1
    int dense_n;   // dofs of the coarsest level when it is inverted densely, else 0
    int degree;    // Chebyshev degree on level 0 (≤ 2 below)
    int pad;
    int64_t nfree;
    CtaLevel lv[kCtaMaxLevels];
    const double* kdiag64;
    const float* kdiag32;
    const double* sdiag;
    const double* f;
    const double* hvec;
    double *u, *vstar, *ftmp, *q, *qtmp, *r, *s, *bb, *r64;
    float *r32, *z32, *p32, *Ap32, *e32;
    float* lam;            // [kCtaMaxLevels] λ_max per level (written here)
    gg_uzawa_stats* stats;  // device copy of the problem's statistics
    int32_t* status;
};

struct CtaParams {
    double tolerance, inner_rtol_factor;
    int max_iterations, min_iterations, use_absolute, use_preconditioner, inner_max_iterations, recycle;
};

// ---- block-level helpers -------------------------------------------------------------
// Sum over the block in a fixed order; every thread gets the value.
__device__ __noinline__ double cta_sum(double v) {
    __shared__ double s_red[32];
    __shared__ double s_tot;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? s_red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) s_tot = v;
    }
    __syncthreads();
    v = s_tot;
    __syncthreads();
    return v;
}

// Vectors written inside the launch are read with plain (L1-cached) loads: every value a
// thread reads was written by a thread of the same CTA before a block barrier, which makes
// it visible in L1; no read-only (non-coherent) load touches them.
template <typename T>
__device__ __forceinline__ T ldg_cg(const T* p) { return __ldca(p); }

__device__ __forceinline__ bool is_fixed(const uint8_t* bc, int64_t i, int64_t nnode) {
    const int c = (int)(i / nnode);
    return (bc[i - (int64_t)c * nnode] >> c) & 1;
}

// y += K x over the element parity classes (y zero on entry for a fresh product); block
// barriers between classes.  Returns this thread's Σ x_eᵀ K_e x_e when kEnergy.
template <int DIM, typename R, bool kEnergy>
__device__ __noinline__ double cta_apply(const MeshK& mk, const R* mom, const uint8_t* bc, const R* x, R* y) {
    double en = 0.0;
    for (int color = 0; color < (1 << DIM); color++) {
        const int px = color & 1, py = (color >> 1) & 1, pz = DIM == 3 ? (color >> 2) & 1 : 0;
        const int c0 = (mk.n[0] - px + 1) >> 1, c1 = (mk.n[1] - py + 1) >> 1;
        const int c2 = DIM == 3 ? (mk.n[2] - pz + 1) >> 1 : 1;
        const int ncls = c0 * c1 * c2;
        for (int idx = threadIdx.x; idx < ncls; idx += blockDim.x) {
            const int ci = idx % c0, rr = idx / c0;
            const int cj = rr % c1, ck = rr / c1;
            const int i = 2 * ci + px, j = 2 * cj + py, k = DIM == 3 ? 2 * ck + pz : 0;
            en += element_apply_scatter<DIM, R, 2, kEnergy>(mk, mom, bc, x, y, i, j, k,
                                                            i + mk.n[0] * (j + mk.n[1] * k));
        }
        __syncthreads();
    }
    return en;
}

template <typename R>
__device__ void cta_zero(R* v, int64_t n) {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) v[i] = R(0);
}

// y = G p on velocity nodes (node gather), BC rows zero (k_apply_G)
template <int DIM>
__device__ __noinline__ void cta_apply_G(const MeshK& mk, const uint8_t* bc, const double* p, double* y) {
    const int64_t nnode = mk.nnode;
    for (int64_t n = threadIdx.x; n < nnode; n += blockDim.x) {
        const int i = (int)(n % mk.nn[0]);
        const int j = (int)((n / mk.nn[0]) % mk.nn[1]);
        const int k = DIM == 3 ? (int)(n / ((int64_t)mk.nn[0] * mk.nn[1])) : 0;
        double acc[DIM];
#pragma unroll
        for (int c = 0; c < DIM; c++) acc[c] = 0.0;
#pragma unroll
        for (int a = 0; a < (1 << DIM); a++) {
            const int ei = i - (a & 1), ej = j - ((a >> 1) & 1), ek = DIM == 3 ? k - ((a >> 2) & 1) : 0;
            if (ei < 0 || ej < 0 || ek < 0 || ei >= mk.n[0] || ej >= mk.n[1] || (DIM == 3 && ek >= mk.n[2])) continue;
            const double pv = ldg_cg(&p[ei + (int64_t)mk.n[0] * (ej + (int64_t)mk.n[1] * ek)]);
#pragma unroll
            for (int c = 0; c < DIM; c++) acc[c] += mk.Ge[a][c] * pv;
        }
        const uint8_t bm = bc[n];
#pragma unroll
        for (int c = 0; c < DIM; c++) y[(int64_t)c * nnode + n] = ((bm >> c) & 1) ? 0.0 : acc[c];
    }
}

// q = Gᵀ u per element (k_apply_GT)
template <int DIM>
__device__ __noinline__ void cta_apply_GT(const MeshK& mk, const double* u, double* q) {
    for (int64_t e = threadIdx.x; e < mk.nel; e += blockDim.x) {
        int ijk[3];
        elem_ijk(mk, e, ijk);
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < (1 << DIM); a++) {
            const int64_t n = elem_node<DIM>(mk, ijk, a);
#pragma unroll
            for (int c = 0; c < DIM; c++) s += mk.Ge[a][c] * ldg_cg(&u[(int64_t)c * mk.nnode + n]);
        }
        q[e] = s;
    }
}

// ---- multigrid set-up, per level ----------------------------------------------------------
__device__ __forceinline__ double tcoef_c(int a, int ap, double o) {
    if (a == 0) return ap == 0 ? 1.0 : 0.0;
    if (a == 1) return ap == 0 ? 0.5 * o : (ap == 1 ? 0.5 : 0.0);
    return ap == 0 ? 0.25 : (ap == 1 ? 0.5 * o : 0.25);
}

// coarse moments as the exact re-expansion of the children's (k_coarsen_moments)
template <int DIM>
__device__ __noinline__ void cta_coarsen(const MeshK& fk, const MeshK& ck, const double* mf, double* mc, float* mc32) {
    constexpr int NM = n_moments<DIM>();
    for (int64_t E = threadIdx.x; E < ck.nel; E += blockDim.x) {
        const int I = (int)(E % ck.n[0]);
        const int64_t rr = E / ck.n[0];
        const int J = (int)(rr % ck.n[1]), K = (int)(rr / ck.n[1]);
        double acc[NM];
#pragma unroll
        for (int q = 0; q < NM; q++) acc[q] = 0.0;
        for (int ch = 0; ch < (1 << DIM); ch++) {
            const int dx = ch & 1, dy = (ch >> 1) & 1, dz = DIM == 3 ? (ch >> 2) & 1 : 0;
            const int64_t fe = (2 * I + dx) + (int64_t)fk.n[0] * ((2 * J + dy) + (int64_t)fk.n[1] * (2 * K + dz));
            const double ox = 2.0 * dx - 1.0, oy = 2.0 * dy - 1.0, oz = 2.0 * dz - 1.0;
            double f[NM];
#pragma unroll
            for (int q = 0; q < NM; q++) f[q] = ldg_cg(&mf[(int64_t)q * fk.nel + fe]);
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
                                    s += tcoef_c(a, ap, ox) * tcoef_c(b, bp, oy) * (DIM == 3 ? tcoef_c(c, cp, oz) : 1.0) *
                                         f[si];
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

// coarse node (I,J,K) ↔ fine node (2I,2J,2K) (k_coarse_bcmask)
__device__ void cta_coarse_bc(const MeshK& fk, const MeshK& ck, const uint8_t* bf, uint8_t* bcc) {
    for (int64_t N = threadIdx.x; N < ck.nnode; N += blockDim.x) {
        const int I = (int)(N % ck.nn[0]);
        const int64_t rr = N / ck.nn[0];
        const int J = (int)(rr % ck.nn[1]), K = (int)(rr / ck.nn[1]);
        bcc[N] = ldg_cg(&bf[2 * I + (int64_t)fk.nn[0] * (2 * J + (int64_t)fk.nn[1] * 2 * K)]);
    }
}

// Jacobi diagonal of a level from its moments (k_level_diag), summed over the parity
// classes (fixed order); diag must be zero on entry
template <int DIM>
__device__ __noinline__ void cta_level_diag(const MeshK& mk, const double* mom, float* diag) {
    constexpr int NM = n_moments<DIM>();
    for (int color = 0; color < (1 << DIM); color++) {
        const int px = color & 1, py = (color >> 1) & 1, pz = DIM == 3 ? (color >> 2) & 1 : 0;
        const int c0 = (mk.n[0] - px + 1) >> 1, c1 = (mk.n[1] - py + 1) >> 1;
        const int c2 = DIM == 3 ? (mk.n[2] - pz + 1) >> 1 : 1;
        for (int idx = threadIdx.x; idx < c0 * c1 * c2; idx += blockDim.x) {
            const int ci = idx % c0, rr = idx / c0;
            int ijk[3] = {2 * ci + px, 2 * (rr % c1) + py, DIM == 3 ? 2 * (rr / c1) + pz : 0};
            const int64_t e = ijk[0] + (int64_t)mk.n[0] * (ijk[1] + (int64_t)mk.n[1] * ijk[2]);
            double M[NM];
#pragma unroll
            for (int q = 0; q < NM; q++) M[q] = ldg_cg(&mom[(int64_t)q * mk.nel + e]);
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
                                    if (o >= DIM || o == d) {
                                        if (ex[o] != 0) ok = false;
                                        continue;
                                    }
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
                for (int c = 0; c < DIM; c++) {
                    float* dp = &diag[(int64_t)c * mk.nnode + n];
                    *dp = ldg_cg(dp) + (float)(tot + S[c]);
                }
            }
        }
        __syncthreads();
    }
}

__device__ void cta_invert_diag(int64_t n, int64_t nnode, const uint8_t* bc, const float* diag, float* inv) {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
        inv[i] = is_fixed(bc, i, nnode) ? 0.f : 1.f / ldg_cg(&diag[i]);
}

// λ_max(D⁻¹A) by power steps from a hashed start (k_hash_fill, k_power_step, k_power_norm)
template <int DIM>
__device__ __noinline__ float cta_power(const CtaLevel& L) {
    const int64_t n = (int64_t)DIM * L.mk.nnode;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        uint32_t h = (uint32_t)i * 2654435761u + 0x9e3779b9u;
        h ^= h >> 15;
        h *= 0x85ebca6bu;
        h ^= h >> 13;
        L.x[i] = is_fixed(L.bc, i, L.mk.nnode) ? 0.f : ((float)(h & 0xffffff) / 16777216.f - 0.5f);
        L.t[i] = 0.f;
    }
    __syncthreads();
    double lam = 1.0;
    for (int step = 0; step < kCtaPowerSteps; step++) {
        cta_apply<DIM, float, false>(L.mk, L.mom32, L.bc, L.x, L.t);
        double yy = 0.0, xx = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const float v = L.invd[i] * ldg_cg(&L.t[i]);
            const float xv = ldg_cg(&L.x[i]);
            L.r[i] = v;
            L.t[i] = 0.f;
            yy += (double)v * v;
            xx += (double)xv * xv;
        }
        yy = cta_sum(yy);
        xx = cta_sum(xx);
        if (xx <= 0.0 || yy <= 0.0) break;
        lam = sqrt(yy / xx);
        const float sc = (float)(1.0 / sqrt(yy));
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) L.x[i] = sc * ldg_cg(&L.r[i]);
        __syncthreads();
    }
    return (float)lam;
}

// dense operator of the coarsest level (free-free block, identity on BC dofs) into shared
// memory, by the apply's element arithmetic on unit vectors, then inverted in place
// (Gauss–Jordan without pivoting: the matrix is symmetric positive definite)
template <int DIM>
__device__ __noinline__ void cta_dense_inverse(const CtaLevel& L, int n, float* A) {
    constexpr int NS = 1 << DIM;
    constexpr int NM = n_moments<DIM>();
    const MeshK& mk = L.mk;
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) A[i] = 0.f;
    __syncthreads();
    // one (element, local dof) pair per thread and pass; columns accumulate with shared
    // atomics (pairs of one class never share a node, classes are separated by barriers)
    for (int color = 0; color < NS; color++) {
        const int px = color & 1, py = (color >> 1) & 1, pz = DIM == 3 ? (color >> 2) & 1 : 0;
        const int c0 = (mk.n[0] - px + 1) >> 1, c1 = (mk.n[1] - py + 1) >> 1;
        const int c2 = DIM == 3 ? (mk.n[2] - pz + 1) >> 1 : 1;
        const int ncls = c0 * c1 * c2;
        for (int w = threadIdx.x; w < ncls * NS * DIM; w += blockDim.x) {
            const int idx = w / (NS * DIM), ldof = w % (NS * DIM);
            const int ca = ldof / DIM, cc = ldof % DIM;  // unit vector at corner ca, component cc
            const int ci = idx % c0, rr = idx / c0;
            const int i = 2 * ci + px, j = 2 * (rr % c1) + py, k = DIM == 3 ? 2 * (rr / c1) + pz : 0;
            const int32_t nn0 = mk.nn[0], nn01 = mk.nn[0] * mk.nn[1];
            const int32_t n0 = i + nn0 * j + (DIM == 3 ? nn01 * k : 0);
            const int32_t node = local_node<DIM>(n0, nn0, nn01, ca);
            const int col = cc * (int)mk.nnode + node;
            if ((L.bc[node] >> cc) & 1) continue;
            float m[DIM][NS];
#pragma unroll
            for (int c = 0; c < DIM; c++)
#pragma unroll
                for (int a = 0; a < NS; a++) m[c][a] = (c == cc && a == ca) ? 1.f : 0.f;
            float M[NM];
            const int64_t e = i + (int64_t)mk.n[0] * (j + (int64_t)mk.n[1] * k);
#pragma unroll
            for (int q = 0; q < NM; q++) M[q] = ldg_cg(&L.mom32[(int64_t)q * mk.nel + e]);
            uint32_t fixed = 0;
            constexpr int NR = NS / 2;
#pragma unroll
            for (int q = 0; q < NR; q++) {
                const int32_t ro = (q & 1) * nn0 + (DIM == 3 ? ((q >> 1) & 1) * nn01 : 0);
                fixed |= ((uint32_t)L.bc[n0 + ro] | ((uint32_t)L.bc[n0 + ro + 1] << 4)) << (8 * q);
            }
            // the column: rows c*nnode + node of the element's corners
            element_compute_scatter<DIM, float, false>(mk, m, M, fixed, A + (size_t)col * n, n0);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (is_fixed(L.bc, i, mk.nnode)) A[(size_t)i * n + i] = 1.f;
    __syncthreads();
    // in-place Gauss–Jordan inversion (A symmetric: the column-major build is the matrix):
    // per pivot k, f_i = A[i][k]; row k ← (row k with A[k][k] = 1) / A[k][k]; every other
    // row i ← (row i with A[i][k] = 0) − f_i · row k
    __shared__ float s_col[kCtaDenseMax];
    __shared__ float s_piv;
    for (int kk = 0; kk < n; kk++) {
        for (int ii = threadIdx.x; ii < n; ii += blockDim.x) s_col[ii] = A[(size_t)ii * n + kk];
        if (threadIdx.x == 0) s_piv = 1.f / A[(size_t)kk * n + kk];
        __syncthreads();
        const float piv = s_piv;
        for (int jj = threadIdx.x; jj < n; jj += blockDim.x) {
            const float v = jj == kk ? 1.f : A[(size_t)kk * n + jj];
            A[(size_t)kk * n + jj] = v * piv;
        }
        __syncthreads();
        for (int w = threadIdx.x; w < n * n; w += blockDim.x) {
            const int ii = w / n, jj = w % n;
            if (ii == kk) continue;
            const float old = jj == kk ? 0.f : A[(size_t)ii * n + jj];
            A[(size_t)ii * n + jj] = old - s_col[ii] * A[(size_t)kk * n + jj];
        }
        __syncthreads();
    }
}

// ---- the V-cycle ---------------------------------------------------------------------------
struct CtaCheb {
    float inv_theta, c1[8], c2[8];
};

__device__ CtaCheb cta_cheb(float lam_est, int degree) {
    // cheb_coef (gg_mg.cu): interval [0.1, 1.1]·λ_max
    const double lmax = 1.1 * lam_est, lmin = 0.1 * lam_est;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    const double sigma = theta / delta;
    CtaCheb cc{};
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

// r = b, d = D⁻¹b/θ, x = d, t = 0
__device__ void cta_cheb_start(const CtaLevel& L, int64_t n, const float* b, float* x, float inv_theta) {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float rv = ldg_cg(&b[i]);
        const float dv = inv_theta * L.invd[i] * rv;
        L.r[i] = rv;
        L.d[i] = dv;
        x[i] = dv;
        L.t[i] = 0.f;
    }
    __syncthreads();
}

// r −= t, d = c1 d + c2 D⁻¹ r, x += d, t = 0
__device__ void cta_cheb_step(const CtaLevel& L, int64_t n, float* x, float c1, float c2) {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float rv = ldg_cg(&L.r[i]) - ldg_cg(&L.t[i]);
        const float dv = c1 * ldg_cg(&L.d[i]) + c2 * L.invd[i] * rv;
        L.r[i] = rv;
        L.d[i] = dv;
        x[i] = ldg_cg(&x[i]) + dv;
        L.t[i] = 0.f;
    }
    __syncthreads();
}

// r = b − t, d = D⁻¹ r/θ, x += d, t = 0
__device__ void cta_cheb_restart(const CtaLevel& L, int64_t n, const float* b, float* x, float inv_theta) {
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float rv = ldg_cg(&b[i]) - ldg_cg(&L.t[i]);
        const float dv = inv_theta * L.invd[i] * rv;
        L.r[i] = rv;
        L.d[i] = dv;
        x[i] = ldg_cg(&x[i]) + dv;
        L.t[i] = 0.f;
    }
    __syncthreads();
}

// b_C = Pᵀ (r − t)_F, zero on coarse BC dofs (k_restrict / phase_restrict)
template <int DIM>
__device__ __noinline__ void cta_restrict(const CtaLevel& F, const CtaLevel& C) {
    const MeshK& fk = F.mk;
    const MeshK& ck = C.mk;
    for (int64_t N = threadIdx.x; N < ck.nnode; N += blockDim.x) {
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
                    for (int c = 0; c < DIM; c++) {
                        const int64_t q = (int64_t)c * fk.nnode + n;
                        acc[c] += w * (ldg_cg(&F.r[q]) - ldg_cg(&F.t[q]));
                    }
                }
        const uint8_t bm = C.bc[N];
#pragma unroll
        for (int c = 0; c < DIM; c++) C.b[(int64_t)c * ck.nnode + N] = ((bm >> c) & 1) ? 0.f : acc[c];
    }
    __syncthreads();
}

// x_F += P x_C (fine BC dofs untouched), t_F = 0 (k_prolong_add / phase_prolong)
template <int DIM>
__device__ __noinline__ void cta_prolong(const CtaLevel& F, float* xf, const CtaLevel& C) {
    const MeshK& fk = F.mk;
    const MeshK& ck = C.mk;
    for (int64_t n = threadIdx.x; n < fk.nnode; n += blockDim.x) {
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
            const float w = ((q & 1) ? wh[0] : wl[0]) * ((q & 2) ? wh[1] : wl[1]) *
                            (DIM == 3 ? ((q & 4) ? wh[2] : wl[2]) : 1.f);
            if (w == 0.f) continue;
            const int64_t N = I + (int64_t)ck.nn[0] * (J + (int64_t)ck.nn[1] * K);
#pragma unroll
            for (int c = 0; c < DIM; c++) acc[c] += w * ldg_cg(&C.x[(int64_t)c * ck.nnode + N]);
        }
        const uint8_t bm = F.bc[n];
#pragma unroll
        for (int c = 0; c < DIM; c++) {
            const int64_t q = (int64_t)c * fk.nnode + n;
            if (!((bm >> c) & 1)) xf[q] = ldg_cg(&xf[q]) + acc[c];
            F.t[q] = 0.f;
        }
    }
    __syncthreads();
}

// x = M⁻¹ b on level 0 (b, x: the FCG's residual and preconditioned vector)
template <int DIM>
__device__ __noinline__ void cta_vcycle(const CtaProblem& P, const CtaCheb* cheb, const float* dense, const float* b0, float* x0) {
    const int ns = P.nlevels - 1;  // smoothed levels 0 .. ns−1; level ns is the coarsest
    for (int l = 0; l < ns; l++) {
        const CtaLevel& L = P.lv[l];
        const int64_t n = (int64_t)DIM * L.mk.nnode;
        const float* bl = l == 0 ? b0 : L.b;
        float* xl = l == 0 ? x0 : L.x;
        const int dl = l == 0 ? P.degree : min(P.degree, 2);
        cta_cheb_start(L, n, bl, xl, cheb[l].inv_theta);
        for (int k = 1; k < dl; k++) {
            cta_apply<DIM, float, false>(L.mk, L.mom32, L.bc, L.d, L.t);
            cta_cheb_step(L, n, xl, cheb[l].c1[k], cheb[l].c2[k]);
        }
        cta_apply<DIM, float, false>(L.mk, L.mom32, L.bc, L.d, L.t);
        cta_restrict<DIM>(L, P.lv[l + 1]);
    }
    {
        const CtaLevel& C = P.lv[ns];
        const int64_t n = (int64_t)DIM * C.mk.nnode;
        if (P.dense_n) {  // x = A⁻¹ b, one thread per row
            for (int64_t row = threadIdx.x; row < n; row += blockDim.x) {
                float s = 0.f;
                for (int64_t k = 0; k < n; k++) s += dense[row * n + k] * ldg_cg(&C.b[k]);
                C.x[row] = s;
            }
            __syncthreads();
        } else {  // a long Chebyshev sweep from zero
            cta_cheb_start(C, n, C.b, C.x, cheb[ns].inv_theta);
            for (int k = 1; k < kCtaCoarseChebDegree; k++) {
                cta_apply<DIM, float, false>(C.mk, C.mom32, C.bc, C.d, C.t);
                cta_cheb_step(C, n, C.x, cheb[ns].c1[k], cheb[ns].c2[k]);
            }
        }
    }
    for (int l = ns - 1; l >= 0; l--) {
        const CtaLevel& L = P.lv[l];
        const int64_t n = (int64_t)DIM * L.mk.nnode;
        const float* bl = l == 0 ? b0 : L.b;
        float* xl = l == 0 ? x0 : L.x;
        const int dl = l == 0 ? P.degree : min(P.degree, 2);
        cta_prolong<DIM>(L, xl, P.lv[l + 1]);
        cta_apply<DIM, float, false>(L.mk, L.mom32, L.bc, xl, L.t);
        cta_cheb_restart(L, n, bl, xl, cheb[l].inv_theta);
        for (int k = 1; k < dl; k++) {
            cta_apply<DIM, float, false>(L.mk, L.mom32, L.bc, L.d, L.t);
            cta_cheb_step(L, n, xl, cheb[l].c1[k], cheb[l].c2[k]);
        }
    }
}

// ---- FP32 flexible CG with the V-cycle (fcg_body of gg_fused.cu, one CTA) -------------------
// x = K32⁻¹ b to ‖r‖ ≤ rtol‖b‖; returns 0, 1 (cap reached) or 2 (non-finite); *its
template <int DIM>
__device__ __noinline__ int cta_fcg(const CtaProblem& P, const CtaCheb* cheb, const float* dense, const float* b, float* x,
                       double rtol, int maxit, int* its) {
    const CtaLevel& L0 = P.lv[0];
    const MeshK& mk = L0.mk;
    const int64_t n = (int64_t)DIM * mk.nnode;
    float* r = P.r32;
    float* z = P.z32;
    float* p = P.p32;
    float* Ap = P.Ap32;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float rv = is_fixed(L0.bc, i, mk.nnode) ? 0.f : ldg_cg(&b[i]);
        x[i] = 0.f;
        r[i] = rv;
        p[i] = 0.f;
        Ap[i] = 0.f;
        acc += (double)rv * rv;
    }
    const double rnorm0 = sqrt(cta_sum(acc));
    const double ttol = fmax(rtol * rnorm0, 1e-30);
    *its = 0;
    if (rnorm0 <= ttol) return 0;
    double pAp = 1.0;
    for (int it = 0;;) {
        cta_vcycle<DIM>(P, cheb, dense, r, z);
        double rz = 0.0, zap = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const double zv = ldg_cg(&z[i]);
            rz += (double)ldg_cg(&r[i]) * zv;
            zap += zv * (double)ldg_cg(&Ap[i]);
        }
        rz = cta_sum(rz);
        zap = cta_sum(zap);
        // truncated flexible CG (Notay 2000): β = −(z·Ap)/(pᵀAp), p = z on the first step
        const float beta = it == 0 ? 0.f : (float)(-zap / pAp);
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            p[i] = ldg_cg(&z[i]) + beta * ldg_cg(&p[i]);
            Ap[i] = 0.f;
        }
        __syncthreads();
        pAp = cta_sum(cta_apply<DIM, float, true>(mk, L0.mom32, L0.bc, p, Ap));
        if (!(pAp > 0.0) || isinf(pAp)) return 2;
        const float alpha = (float)(rz / pAp);
        double rr = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            x[i] = ldg_cg(&x[i]) + alpha * ldg_cg(&p[i]);
            const float rv = ldg_cg(&r[i]) - alpha * ldg_cg(&Ap[i]);
            r[i] = rv;
            rr += (double)rv * rv;
        }
        const double rn = sqrt(cta_sum(rr));
        it++;
        *its = it;
        if (!(rn == rn) || isinf(rn)) return 2;
        if (rn <= ttol) return 0;
        if (it >= maxit) return 1;
    }
}

// ‖D⁻¹ r‖ over free rows where r = b − (K x, in r on entry), writing r (k_defect)
__device__ __noinline__ double cta_defect(int64_t n, int64_t nnode, const uint8_t* bc, const double* b, const double* diag,
                             double* r) {
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const bool fixed = is_fixed(bc, i, nnode);
        const double rv = fixed ? 0.0 : ldg_cg(&b[i]) - ldg_cg(&r[i]);
        r[i] = rv;
        const double zv = fixed ? 0.0 : rv / diag[i];
        acc += zv * zv;
    }
    return sqrt(cta_sum(acc));
}

// x = K⁻¹ b: FP64 defect correction around FP32 multigrid FCG sweeps (inner_solve, mixed
// path with multigrid): the reference's stopping rule on the Jacobi-preconditioned FP64
// defect.  Returns a GG status; *its = FCG iterations.
template <int DIM>
__device__ __noinline__ int cta_inner(const CtaProblem& P, const CtaCheb* cheb, const float* dense, const double* b, double* x,
                         double rtol, int maxit, bool warm, bool& tight, int* its) {
    const CtaLevel& L0 = P.lv[0];
    const MeshK& mk = L0.mk;
    const int64_t n = (int64_t)DIM * mk.nnode;
    double* r64 = P.r64;
    if (!warm)
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) x[i] = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) r64[i] = 0.0;
    __syncthreads();
    const double rnorm0 = cta_defect(n, mk.nnode, L0.bc, b, P.kdiag64, r64);
    const double ttol = fmax(rtol * rnorm0, 1e-50);
    *its = 0;
    double rn_cur = rnorm0;
    if (warm) {
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) r64[i] = 0.0;
        __syncthreads();
        cta_apply<DIM, double, false>(mk, L0.mom64, L0.bc, x, r64);
        const double rn = cta_defect(n, mk.nnode, L0.bc, b, P.kdiag64, r64);
        if (!(rn == rn)) return GG_ERR_NONFINITE;
        if (rn <= ttol) return GG_OK;
        rn_cur = rn;
    } else if (rnorm0 <= ttol) {
        return GG_OK;
    }
    const int sweep_cap = min(maxit, 150);
    int total = 0;
    for (int sweep = 0; sweep < 50; sweep++) {
        const double inner_rtol = tight ? 1e-5 : 1e-4;
        const double srtol = fmax(inner_rtol, fmin(0.5, ttol / rn_cur));
        // e = K32⁻¹ (FP32) r; level 0's b (unused by the V-cycle there) holds the FP32 defect
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) P.lv[0].b[i] = (float)ldg_cg(&r64[i]);
        __syncthreads();
        int it = 0;
        const int frc = cta_fcg<DIM>(P, cheb, dense, P.lv[0].b, P.e32, srtol, sweep_cap, &it);
        total += it;
        if (frc == 2) {
            *its = total;
            return GG_ERR_NONFINITE;
        }
        // x += e ; r = b − K64 x
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            x[i] = ldg_cg(&x[i]) + (double)ldg_cg(&P.e32[i]);
            r64[i] = 0.0;
        }
        __syncthreads();
        cta_apply<DIM, double, false>(mk, L0.mom64, L0.bc, x, r64);
        const double rn = cta_defect(n, mk.nnode, L0.bc, b, P.kdiag64, r64);
        if (!(rn == rn)) {
            *its = total;
            return GG_ERR_NONFINITE;
        }
        if (sweep >= 2) tight = true;
        if (rn <= ttol) {
            *its = total;
            return GG_OK;
        }
        rn_cur = rn;
        if (total >= maxit) break;
    }
    *its = total;
    return GG_ERR_NOT_CONVERGED;
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// One whole problem: multigrid set-up, then _Stokes_SLE_UzawaSolver_Solve
// (Stokes_SLE_UzawaSolver.cxx:393-938) as gg_solve.cu:uzawa_solve does it.
template <int DIM>
__device__ __noinline__ void cta_solve_problem(const CtaProblem& P, const CtaParams& prm, float* dense) {
    __shared__ CtaCheb s_cheb[kCtaMaxLevels];
    const uint64_t t_start = globaltimer();
    // ---- multigrid set-up
    const int nl = P.nlevels;
    {
        const CtaLevel& L0 = P.lv[0];
        cta_invert_diag((int64_t)DIM * L0.mk.nnode, L0.mk.nnode, L0.bc, P.kdiag32, L0.invd);
    }
    for (int l = 1; l < nl; l++) {
        const CtaLevel& F = P.lv[l - 1];
        const CtaLevel& L = P.lv[l];
        const int64_t n = (int64_t)DIM * L.mk.nnode;
        cta_coarse_bc(F.mk, L.mk, F.bc, L.bc);
        cta_coarsen<DIM>(F.mk, L.mk, F.mom64, L.mom64, L.mom32);
        cta_zero(L.t, n);
        __syncthreads();
        cta_level_diag<DIM>(L.mk, L.mom64, L.t);
        cta_invert_diag(n, L.mk.nnode, L.bc, L.t, L.invd);
        __syncthreads();
    }
    __syncthreads();
    for (int l = 0; l < nl; l++) {
        const bool coarsest = l == nl - 1;
        if (coarsest && P.dense_n) break;
        const float lam = cta_power<DIM>(P.lv[l]);
        if (threadIdx.x == 0) {
            const int deg = coarsest ? kCtaCoarseChebDegree : (l == 0 ? P.degree : min(P.degree, 2));
            s_cheb[l] = cta_cheb(lam, deg);
            P.lam[l] = lam;
        }
        __syncthreads();
    }
    if (P.dense_n) cta_dense_inverse<DIM>(P.lv[nl - 1], P.dense_n, dense);
    __syncthreads();

    // ---- Uzawa
    const CtaLevel& L0 = P.lv[0];
    const MeshK& mk = L0.mk;
    const int64_t nd = (int64_t)DIM * mk.nnode, ne = mk.nel;
    const double scaleq = sqrt((double)ne);
    const int maxit = prm.inner_max_iterations > 0 ? prm.inner_max_iterations : 10000;
    int status = GG_OK, it = 0, inner_total = 0, inner_solves = 0;
    bool tight = false;
    double relres = 0.0, absres = 0.0;
    auto inner = [&](const double* b, double* x, double rtol, bool warm) {
        int its = 0;
        const int rc = cta_inner<DIM>(P, s_cheb, dense, b, x, rtol, maxit, warm, tight, &its);
        inner_total += its;
        inner_solves++;
        return rc;
    };
    double fn = 0.0;
    for (int64_t i = threadIdx.x; i < nd; i += blockDim.x) fn += P.f[i] * P.f[i];
    const double fnorm = sqrt(cta_sum(fn));
    if (fnorm / sqrt((double)P.nfree) <= 1e-99) {
        status = GG_ERR_ZERO_FORCE;
    } else {
        // STEP 1 (:553-565)
        status = inner(P.f, P.vstar, prm.tolerance, false);
        double rs = 0.0;
        if (status == GG_OK) {
            cta_apply_GT<DIM>(mk, P.vstar, P.qtmp);
            __syncthreads();
            for (int64_t e = threadIdx.x; e < ne; e += blockDim.x) {
                const double v = ldg_cg(&P.qtmp[e]) - P.hvec[e];
                P.qtmp[e] = v;
                rs += v * v;
            }
        }
        const double rhs_scale = sqrt(cta_sum(rs)) / scaleq;
        const double inner_rtol = prm.inner_rtol_factor * prm.tolerance;
        if (status == GG_OK && !isfinite(rhs_scale)) status = GG_ERR_NONFINITE;
        // STEP 3 (:616-659): u = K⁻¹(f − G q), r = Gᵀu − h
        if (status == GG_OK) {
            cta_apply_G<DIM>(mk, L0.bc, P.q, P.ftmp);
            __syncthreads();
            for (int64_t i = threadIdx.x; i < nd; i += blockDim.x) P.ftmp[i] = P.f[i] - ldg_cg(&P.ftmp[i]);
            __syncthreads();
            status = inner(P.ftmp, P.u, inner_rtol, false);
        }
        bool exact = false;
        if (status == GG_OK) {
            cta_apply_GT<DIM>(mk, P.u, P.r);
            __syncthreads();
            double r0 = 0.0, uu = 0.0, hh = 0.0;
            for (int64_t e = threadIdx.x; e < ne; e += blockDim.x) {
                const double v = ldg_cg(&P.r[e]) - P.hvec[e];
                P.r[e] = v;
                r0 += v * v;
                hh += P.hvec[e] * P.hvec[e];
            }
            for (int64_t i = threadIdx.x; i < nd; i += blockDim.x) uu += ldg_cg(&P.u[i]) * ldg_cg(&P.u[i]);
            r0 = sqrt(cta_sum(r0));
            uu = sqrt(cta_sum(uu));
            hh = sqrt(cta_sum(hh));
            // a velocity that meets the constraint to rounding ends the solve (as uzawa_solve)
            double gmax = 0.0;
            for (int a = 0; a < (1 << DIM); a++)
                for (int c = 0; c < DIM; c++) gmax = fmax(gmax, fabs(mk.Ge[a][c]));
            if (r0 <= 64.0 * 2.220446049250313e-16 * (gmax * sqrt((double)(1 << DIM)) * uu + hh)) {
                exact = true;
                absres = r0 / scaleq;
            }
        }
        // STEP 4 (:664-837)
        double zr_prev = 1.0;
        while (status == GG_OK && !exact) {
            double zr = 0.0;
            for (int64_t e = threadIdx.x; e < ne; e += blockDim.x) {
                const double rv = ldg_cg(&P.r[e]);
                const double zv = prm.use_preconditioner ? rv / P.sdiag[e] : rv;
                P.qtmp[e] = zv;
                zr += zv * rv;
            }
            zr = cta_sum(zr);
            const double beta = it == 0 ? 0.0 : zr / zr_prev;
            for (int64_t e = threadIdx.x; e < ne; e += blockDim.x)
                P.s[e] = ldg_cg(&P.qtmp[e]) + (it == 0 ? 0.0 : beta * ldg_cg(&P.s[e]));
            __syncthreads();
            cta_apply_G<DIM>(mk, L0.bc, P.s, P.ftmp);
            const bool warm = prm.recycle && it > 0;
            if (warm)
                for (int64_t i = threadIdx.x; i < nd; i += blockDim.x) P.vstar[i] = beta * ldg_cg(&P.vstar[i]);
            __syncthreads();
            status = inner(P.ftmp, P.vstar, inner_rtol, warm);
            if (status != GG_OK) break;
            cta_apply_GT<DIM>(mk, P.vstar, P.qtmp);
            __syncthreads();
            double sq = 0.0;
            for (int64_t e = threadIdx.x; e < ne; e += blockDim.x) sq += ldg_cg(&P.s[e]) * ldg_cg(&P.qtmp[e]);
            sq = cta_sum(sq);
            const double alpha = zr / sq;
            if (!isfinite(zr) || !isfinite(sq) || !isfinite(alpha)) {
                status = GG_ERR_NONFINITE;
                break;
            }
            double rr = 0.0;
            for (int64_t e = threadIdx.x; e < ne; e += blockDim.x) {
                P.q[e] = ldg_cg(&P.q[e]) + alpha * ldg_cg(&P.s[e]);
                const double rv = ldg_cg(&P.r[e]) - alpha * ldg_cg(&P.qtmp[e]);
                P.r[e] = rv;
                rr += rv * rv;
            }
            for (int64_t i = threadIdx.x; i < nd; i += blockDim.x) P.u[i] = ldg_cg(&P.u[i]) - alpha * ldg_cg(&P.vstar[i]);
            zr_prev = zr;
            absres = sqrt(cta_sum(rr)) / scaleq;
            relres = absres / rhs_scale;
            if (!isfinite(absres)) {
                status = GG_ERR_NONFINITE;
                break;
            }
            if (!(it < prm.max_iterations)) {
                status = GG_ERR_NOT_CONVERGED;
                it++;
                break;
            }
            it++;
            const double chosen = prm.use_absolute ? absres : relres;
            if (!((chosen > prm.tolerance) || (it < prm.min_iterations))) break;
        }
        if (exact) relres = 0.0;
    }
    __syncthreads();
    const uint64_t t_end = globaltimer();
    // summary norms (:844-877): |Gᵀu|/|u| and |f − K u − G q|/|f|
    cta_apply_GT<DIM>(mk, P.u, P.qtmp);
    cta_apply_G<DIM>(mk, L0.bc, P.q, P.vstar);
    for (int64_t i = threadIdx.x; i < nd; i += blockDim.x) P.ftmp[i] = 0.0;
    __syncthreads();
    cta_apply<DIM, double, false>(mk, L0.mom64, L0.bc, P.u, P.ftmp);
    double dv = 0.0, uu = 0.0, mr = 0.0;
    for (int64_t e = threadIdx.x; e < ne; e += blockDim.x) dv += ldg_cg(&P.qtmp[e]) * ldg_cg(&P.qtmp[e]);
    for (int64_t i = threadIdx.x; i < nd; i += blockDim.x) {
        uu += ldg_cg(&P.u[i]) * ldg_cg(&P.u[i]);
        const double m = P.f[i] - ldg_cg(&P.ftmp[i]) - ldg_cg(&P.vstar[i]);
        mr += m * m;
    }
    dv = sqrt(cta_sum(dv));
    uu = sqrt(cta_sum(uu));
    mr = sqrt(cta_sum(mr));
    if (threadIdx.x == 0) {
        gg_uzawa_stats S;
        memset(&S, 0, sizeof S);
        S.outer_iterations = it;
        S.inner_iterations = inner_total;
        S.inner_solves = inner_solves;
        S.rel_residual = relres;
        S.abs_residual = absres;
        S.div_u = uu > 0 ? dv / uu : 0.0;
        S.momentum_residual = fnorm > 0 ? mr / fnorm : 0.0;
        S.solve_ms = (double)(t_end - t_start) * 1e-6;
        *P.stats = S;
        *P.status = status;
    }
    __syncthreads();
}

template <int DIM>
__global__ void __launch_bounds__(cta_threads<DIM>(), 1)
k_batch_uzawa(const CtaProblem* __restrict__ probs, const int32_t* __restrict__ order, int n, CtaParams prm,
              int* next) {
    extern __shared__ float s_dense[];
    __shared__ int s_p;
    for (;;) {
        if (threadIdx.x == 0) s_p = atomicAdd(next, 1);
        __syncthreads();
        const int pi = s_p;
        __syncthreads();
        if (pi >= n) return;
        cta_solve_problem<DIM>(probs[order[pi]], prm, s_dense);
    }
}

}  // namespace

// ---- host side ------------------------------------------------------------------------------
// Whether the batched CTA solver takes these parameters: the mixed path with the multigrid
// inner solve (the learned variants fall back to it: no network runs inside a CTA).
bool cta_batch_supported(const gg_uzawa_params& prm) {
    return prm.precision == GG_PRECISION_MIXED &&
           (prm.inner == GG_INNER_MG_CG || prm.inner == GG_INNER_LEARNED_CG);
}

// Levels of a problem for the CTA solver: halve while every axis is even and ≥ 4 elements
// and the level has more than kCtaDenseMax dofs; the coarsest is inverted densely when it
// has at most kCtaDenseMax dofs.
static void cta_levels(Handle& H, std::vector<MeshK>& mks, int& dense_n) {
    mks.clear();
    mks.push_back(H.mk);
    for (;;) {
        const MeshK& f = mks.back();
        if ((int64_t)H.dim * f.nnode <= kCtaDenseMax) break;
        bool can = mks.size() < (size_t)kCtaMaxLevels;
        for (int d = 0; d < H.dim; d++)
            if (f.n[d] % 2 != 0 || f.n[d] < kCtaMinCoarse) can = false;
        if (!can) break;
        gg_mesh_desc cd{};
        cd.dim = H.dim;
        for (int d = 0; d < H.dim; d++) {
            cd.elements[d] = f.n[d] / 2;
            cd.min[d] = f.min[d];
            cd.max[d] = f.max[d];
        }
        mks.push_back(make_mesh(cd));
    }
    const int64_t nc = (int64_t)H.dim * mks.back().nnode;
    dense_n = (mks.size() > 1 && nc <= kCtaDenseMax) ? (int)nc : 0;
}

// Solve every problem (located and built with the FP32 moments) in one launch.  status[i]
// and stats[i] per problem; u_out / p_out host arrays (nodal velocity with its boundary
// values, element pressure).  Returns GG_OK when the launch ran (per-problem failures are
// in status), or a CUDA / invalid-argument status.
int cta_batch_solve(std::vector<Handle*>& hs, const gg_uzawa_params& prm, double* const* u_out,
                    double* const* p_out, gg_uzawa_stats* stats, int32_t* status) {
    const int n = (int)hs.size();
    const int dim = hs[0]->dim;
    for (Handle* H : hs)
        if (H->dim != dim) return GG_ERR_INVALID;
    std::vector<CtaProblem> probs(n);
    for (int i = 0; i < n; i++) {
        Handle& H = *hs[i];
        CtaProblem& P = probs[i];
        std::memset(&P, 0, sizeof P);
        std::vector<MeshK> mks;
        int dense_n = 0;
        cta_levels(H, mks, dense_n);
        P.nlevels = (int)mks.size();
        P.dense_n = dense_n;
        P.degree = prm.smoothing_degree > 0 ? prm.smoothing_degree : 2;
        if (P.degree < 2 || P.degree > 4) return GG_ERR_INVALID;
        P.nfree = H.nfree;
        // storage: the handle's FP32/FP64 solver vectors and its own level buffers
        const int64_t nd = H.ndof, ne = H.nel;
        for (DBuf* b : {&H.u, &H.vstar, &H.ftmp, &H.cg_b, &H.cg_r}) b->ensure(sizeof(double) * nd);
        for (DBuf* b : {&H.q, &H.qtmp, &H.r, &H.s}) b->ensure(sizeof(double) * ne);
        for (DBuf* b : {&H.r32, &H.z32, &H.p32, &H.Ap32, &H.e32}) b->ensure(sizeof(float) * nd);
        H.cta_levels.resize(P.nlevels);
        for (int l = 0; l < P.nlevels; l++) {
            if (!H.cta_levels[l]) H.cta_levels[l] = std::make_unique<MGLevel>();
            MGLevel& M = *H.cta_levels[l];
            M.mk = mks[l];
            const int64_t lnd = (int64_t)dim * mks[l].nnode;
            for (DBuf* b : {&M.x, &M.b, &M.r, &M.d, &M.t, &M.invdiag}) b->ensure(sizeof(float) * lnd);
            CtaLevel& L = P.lv[l];
            L.mk = mks[l];
            if (l == 0) {
                L.mom64 = H.mom64.as<double>();
                L.mom32 = H.mom32.as<float>();
                L.bc = H.bcmask.as<uint8_t>();
            } else {
                M.own_mom64.ensure(sizeof(double) * H.nm * mks[l].nel);
                M.own_mom32.ensure(sizeof(float) * H.nm * mks[l].nel);
                M.own_bcmask.ensure(mks[l].nnode);
                L.mom64 = M.own_mom64.as<double>();
                L.mom32 = M.own_mom32.as<float>();
                L.bc = M.own_bcmask.as<uint8_t>();
            }
            L.invd = M.invdiag.as<float>();
            L.x = M.x.as<float>();
            L.b = M.b.as<float>();
            L.r = M.r.as<float>();
            L.d = M.d.as<float>();
            L.t = M.t.as<float>();
        }
        H.cta_lam.ensure(sizeof(float) * kCtaMaxLevels);
        P.kdiag64 = H.kdiag64.as<double>();
        P.kdiag32 = H.kdiag32.as<float>();
        P.sdiag = H.sdiag.as<double>();
        P.f = H.f.as<double>();
        P.hvec = H.hvec.as<double>();
        P.u = H.u.as<double>();
        P.vstar = H.vstar.as<double>();
        P.ftmp = H.ftmp.as<double>();
        P.q = H.q.as<double>();
        P.qtmp = H.qtmp.as<double>();
        P.r = H.r.as<double>();
        P.s = H.s.as<double>();
        P.bb = H.cg_b.as<double>();
        P.r64 = H.cg_r.as<double>();
        P.r32 = H.r32.as<float>();
        P.z32 = H.z32.as<float>();
        P.p32 = H.p32.as<float>();
        P.Ap32 = H.Ap32.as<float>();
        P.e32 = H.e32.as<float>();
        P.lam = H.cta_lam.as<float>();
        if (prm.reuse_pressure)
            GG_CUDA(cudaMemcpyAsync(H.q.p, p_out[i], sizeof(double) * ne, cudaMemcpyHostToDevice, H.stream));
        else
            GG_CUDA(cudaMemsetAsync(H.q.p, 0, sizeof(double) * ne, H.stream));
    }
    // largest problems first: the queue then ends on small ones
    std::vector<int32_t> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return hs[a]->nel > hs[b]->nel; });
    GG_CUDA(cudaDeviceSynchronize());  // every handle's build (own streams) is complete
    // one device block for the descriptors, the order, the queue head and the outputs
    const size_t bp = sizeof(CtaProblem) * n, bo = sizeof(int32_t) * n, bs = sizeof(gg_uzawa_stats) * n;
    char* dev = nullptr;
    GG_CUDA(cudaMalloc(&dev, bp + bo + bs + sizeof(int32_t) * n + 256));
    CtaProblem* d_probs = reinterpret_cast<CtaProblem*>(dev);
    int32_t* d_order = reinterpret_cast<int32_t*>(dev + bp);
    gg_uzawa_stats* d_stats = reinterpret_cast<gg_uzawa_stats*>(dev + bp + bo);
    int32_t* d_status = reinterpret_cast<int32_t*>(dev + bp + bo + bs);
    int* d_next = reinterpret_cast<int*>(dev + bp + bo + bs + sizeof(int32_t) * n);
    for (int i = 0; i < n; i++) {
        probs[i].stats = d_stats + i;
        probs[i].status = d_status + i;
    }
    int rc = GG_OK;
    try {
        GG_CUDA(cudaMemcpy(d_probs, probs.data(), bp, cudaMemcpyHostToDevice));
        GG_CUDA(cudaMemcpy(d_order, order.data(), bo, cudaMemcpyHostToDevice));
        GG_CUDA(cudaMemset(d_next, 0, sizeof(int)));
        const size_t smem = sizeof(float) * kCtaDenseMax * kCtaDenseMax;
        const void* fn = dim == 2 ? (const void*)k_batch_uzawa<2> : (const void*)k_batch_uzawa<3>;
        GG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int threads = dim == 2 ? cta_threads<2>() : cta_threads<3>();
        int per_sm = 0;
        GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
        int grid = std::max(1, per_sm) * num_sms();
        if (grid > n) grid = n;
        CtaParams cp{};
        cp.tolerance = prm.tolerance;
        cp.inner_rtol_factor = prm.inner_rtol_factor;
        cp.max_iterations = prm.max_iterations;
        cp.min_iterations = prm.min_iterations;
        cp.use_absolute = prm.use_absolute_tolerance;
        cp.use_preconditioner = prm.use_preconditioner;
        cp.inner_max_iterations = prm.inner_max_iterations;
        cp.recycle = prm.recycle_directions;
        cudaEvent_t e0, e1;
        GG_CUDA(cudaEventCreate(&e0));
        GG_CUDA(cudaEventCreate(&e1));
        GG_CUDA(cudaEventRecord(e0, 0));
        if (dim == 2)
            k_batch_uzawa<2><<<grid, threads, smem, 0>>>(d_probs, d_order, n, cp, d_next);
        else
            k_batch_uzawa<3><<<grid, threads, smem, 0>>>(d_probs, d_order, n, cp, d_next);
        GG_CUDA(cudaGetLastError());
        GG_CUDA(cudaEventRecord(e1, 0));
        GG_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        GG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        std::vector<gg_uzawa_stats> hst(n);
        GG_CUDA(cudaMemcpy(hst.data(), d_stats, bs, cudaMemcpyDeviceToHost));
        GG_CUDA(cudaMemcpy(status, d_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; i++) {
            Handle& H = *hs[i];
            hst[i].kernel_launches = 1;
            hst[i].fused_launches = 1;
            hst[i].fused_ms = ms;  // the one launch that solved the batch
            if (stats) stats[i] = hst[i];
            download_solution(H, u_out[i], p_out[i]);
            H.last_solve_ms = hst[i].solve_ms;
        }
    } catch (const CudaError& ce) {
        hs[0]->err = ce.what;
        rc = GG_ERR_CUDA;
    }
    cudaFree(dev);
    return rc;
}

}  // namespace gg
