// gg_dvc.cu -- discrete-Voronoi integration weights (DVCWeights) and population control
// (PCDVC) on sm_100a.
//
// Reference: PICellerator/Weights/src/DVCWeights.cxx:202-953 (grid, region growth,
// centroids) and PICellerator/Utils/src/PCDVC.cxx:656-1512 (split / delete).  Per element
// the reference grows a discrete Voronoi diagram on a res^dim grid of [-1,1]^dim:
//   * seeds: point i takes the grid cell it lies in (a later point overwrites);
//   * passes: point after point, i contests every cell of its boundary list -- an unowned
//     cell is taken, an owned one only when i is strictly closer to its centre -- and
//     rebuilds its boundary list from the neighbours (S, N, E, W, U, D) of the cells it
//     just took that it does not own; passes repeat until one claims nothing;
//   * centroid of i = mean centre of its cells, weight = cells × cell volume.
// B200 mapping: one warp per element, the grid and the boundary lists in shared memory.
// The points stay sequential, as in the reference, but within one point's turn the
// claims and the boundary are sets: a cell's claim depends only on its current owner, and
// the boundary is the set of neighbours of the new claims not owned by the point.  So a
// point's turn runs across the 32 lanes (ballot compaction, a per-turn stamp
// deduplicates the boundary) and gives the reference's ownership exactly.  Centroids are
// summed per point in grid-cell order (one lane per point), the reference's order.
//
// Population control (lane 0, a few dozen items per element): the split list in list
// order; the delete list sorted by decreasing point index; the limits and the interface
// rule of PCDVC.cxx:954-1013; new points appended to the element list, deletions by swap
// with the list's last entry (Swarm_RemoveParticleFromCell, StgDomain/Swarm/src/
// SwarmClass.cxx:976-992); then a new diagram for the element.  The global point arrays
// are rebuilt afterwards (survivors in their order, then the new points), re-located,
// and the integration points of the final diagrams are applied.  The reference's
// swap-with-last reuse of global particle slots is a storage detail that no element's
// list order depends on, and is not reproduced.
//
// Arithmetic follows the reference's double operations one rounding at a time
// (__dadd_rn / __dmul_rn / __ddiv_rn, no contraction), so weights and centroids match the
// CPU restatement bit for bit.
#include <math.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"

namespace gg {

namespace {

constexpr int kMaxCells = 1024;  // grid cells per element
constexpr int kMaxPts = 254;     // points per element (owner byte, 255 = unowned)
constexpr int kPool = 3072;      // boundary-list entries per pass
constexpr int kAxis = 64;        // cells per axis
constexpr int kWarps = 3;        // elements per block
constexpr int kMaxPasses = 4096;
constexpr uint8_t kNone = 255;

enum DvcErr : int32_t { kOk = 0, kTooMany = 1, kPoolFull = 2, kPasses = 3, kUnowned = 4, kTooFew = 5 };

struct DvcSmem {
    double xi[kMaxPts][3];
    double cent[kMaxPts][3];
    double cx[kAxis], cy[kAxis], cz[kAxis];
    uint32_t mark[kMaxCells];
    uint16_t claimed[kMaxCells];
    uint16_t pool[2][kPool];
    uint16_t boff[2][kMaxPts], blen[2][kMaxPts];
    uint16_t cnt[kMaxPts];
    int16_t list[kMaxPts];
    int16_t split[kMaxPts];
    int16_t del[kMaxPts];
    uint8_t owner[kMaxCells];
    uint32_t bump[2];
};

struct DvcArgs {
    int dim, nx, ny, nz, ncell;
    double dx, dy, dz, da;
    int64_t nel, np;
    const int32_t* offsets;
    const double* xi_s;     // [dim][np] sorted local coordinates
    const int32_t* mat_s;   // sorted material
    const int32_t* perm;    // sorted → point index (the reference's swarm index)
    double* cent_out;       // [dim][np] final centroid per sorted point
    double* w_out;          // [np]
    uint8_t* keep;          // [np] 0: deleted
    int pc;                 // population control on
    double maxW, minW;
    int max_splits, max_deletions, split_if, delete_if;
    int stride;             // staging slots per element (max(max_splits, 1))
    int32_t* new_parent;    // [nel*stride] sorted index of the parent
    double* new_xi;         // [nel*stride][dim]
    double* new_cent;       // [nel*stride][dim]
    double* new_w;          // [nel*stride]
    int32_t* nsplit;        // [nel]
    int32_t* ndel;          // [nel]
    int32_t* err;           // [2]: first error code, element
};

__device__ __forceinline__ void set_err(const DvcArgs& a, int code, int64_t e) {
    if (atomicCAS(&a.err[0], 0, code) == 0) a.err[1] = (int32_t)e;
}

// DistanceTest (DVCWeights.cxx:629-634): > 0 when point 2 is strictly closer to c0 than 1
template <int DIM>
__device__ __forceinline__ double dist_test(const double* c0, const double* p1, const double* p2) {
    double v = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const double s = __dsub_rn(__dsub_rn(__dadd_rn(p1[d], p2[d]), c0[d]), c0[d]);
        const double t = __dmul_rn(s, __dsub_rn(p1[d], p2[d]));
        v = d == 0 ? t : __dadd_rn(v, t);
    }
    return v;
}

template <int DIM>
__device__ __forceinline__ int neighbour(const DvcArgs& a, int c, int q) {
    const int ci = c % a.nx, cj = (c / a.nx) % a.ny, ck = c / (a.nx * a.ny);
    switch (q) {
        case 0: return cj > 0 ? c - a.nx : -1;               // S
        case 1: return cj < a.ny - 1 ? c + a.nx : -1;        // N
        case 2: return ci < a.nx - 1 ? c + 1 : -1;           // E
        case 3: return ci > 0 ? c - 1 : -1;                  // W
        case 4: return ck < a.nz - 1 ? c + a.nx * a.ny : -1; // U
        default: return ck > 0 ? c - a.nx * a.ny : -1;       // D
    }
}

// The diagram of S.xi[0..n) and each point's centroid and cell count; false on an error
// (already recorded).  All 32 lanes call it.
template <int DIM>
__device__ bool dvc_warp(const DvcArgs& a, DvcSmem& S, int n, int64_t e) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    for (int c = lane; c < a.ncell; c += 32) {
        S.owner[c] = kNone;
        S.mark[c] = 0u;
    }
    __syncwarp();
    uint32_t stamp = 0;
    // seeds and the first boundary lists, point by point (DVCWeights.cxx:693-725); they
    // go to pool 1, which pass 0 reads
    if (lane == 0) {
        S.bump[1] = 0;
        bool ok = true;
        for (int i = 0; i < n && ok; i++) {
            int k = __double2int_rz(__ddiv_rn(__dsub_rn(S.xi[i][0], -1.0), a.dx));
            int j = __double2int_rz(__ddiv_rn(__dsub_rn(S.xi[i][1], -1.0), a.dy));
            int l = DIM == 3 ? __double2int_rz(__ddiv_rn(__dsub_rn(S.xi[i][2], -1.0), a.dz)) : 0;
            if (k == a.nx) k--;
            if (j == a.ny) j--;
            if (DIM == 3 && l == a.nz) l--;
            k = min(max(k, 0), a.nx - 1);
            j = min(max(j, 0), a.ny - 1);
            l = min(max(l, 0), a.nz - 1);
            const int c = k + j * a.nx + l * a.nx * a.ny;
            S.owner[c] = (uint8_t)i;
            const uint32_t start = S.bump[1];
            uint32_t m = 0;
            for (int q = 0; q < 2 * DIM; q++) {
                const int nb = neighbour<DIM>(a, c, q);
                if (nb >= 0 && S.owner[nb] != i) {
                    if (start + m >= (uint32_t)kPool) {
                        ok = false;
                        break;
                    }
                    S.pool[1][start + m++] = (uint16_t)nb;
                }
            }
            S.boff[1][i] = (uint16_t)start;
            S.blen[1][i] = (uint16_t)m;
            S.bump[1] = start + m;
        }
        if (!ok) set_err(a, kPoolFull, e);
        S.bump[0] = ok ? 0u : 0xffffffffu;
    }
    __syncwarp();
    if (S.bump[0] == 0xffffffffu) return false;
    for (int t = 0;; t++) {
        if (t >= kMaxPasses) {
            if (lane == 0) set_err(a, kPasses, e);
            return false;
        }
        const int prod = t & 1, cons = prod ^ 1;
        if (lane == 0) S.bump[prod] = 0;
        __syncwarp();
        int claimed_pass = 0;
        for (int i = 0; i < n; i++) {
            // contest the boundary (ClaimCells, DVCWeights.cxx:260-330)
            const int off = S.boff[cons][i], len = S.blen[cons][i];
            int nclaim = 0;
            for (int base = 0; base < len; base += 32) {
                const int k = base + lane;
                bool take = false;
                int c = -1;
                if (k < len) {
                    c = S.pool[cons][off + k];
                    const int o = S.owner[c];
                    if (o == kNone) {
                        take = true;
                    } else if (o != i) {
                        const double c0[3] = {S.cx[c % a.nx], S.cy[(c / a.nx) % a.ny],
                                              DIM == 3 ? S.cz[c / (a.nx * a.ny)] : 0.0};
                        take = dist_test<DIM>(c0, S.xi[o], S.xi[i]) > 0.0;
                    }
                    if (take) S.owner[c] = (uint8_t)i;
                }
                const unsigned b = __ballot_sync(full, take);
                if (take) S.claimed[nclaim + __popc(b & ((1u << lane) - 1u))] = (uint16_t)c;
                nclaim += __popc(b);
            }
            claimed_pass += nclaim;
            __syncwarp();
            // the new boundary (UpdateBchain, DVCWeights.cxx:420-470) into pool prod
            if (++stamp == 0u) {
                for (int c = lane; c < a.ncell; c += 32) S.mark[c] = 0u;
                stamp = 1;
                __syncwarp();
            }
            const uint32_t start = S.bump[prod];
            uint32_t m = 0;
            bool overflow = false;
            for (int base = 0; base < nclaim; base += 32) {
                const int k = base + lane;
                const int c0 = k < nclaim ? S.claimed[k] : -1;
#pragma unroll
                for (int q = 0; q < 2 * DIM; q++) {
                    const int nb = c0 >= 0 ? neighbour<DIM>(a, c0, q) : -1;
                    bool add = false;
                    if (nb >= 0 && S.owner[nb] != i) add = atomicExch(&S.mark[nb], stamp) != stamp;
                    const unsigned b = __ballot_sync(full, add);
                    if (add) {
                        const uint32_t pos = start + m + __popc(b & ((1u << lane) - 1u));
                        if (pos < (uint32_t)kPool) S.pool[prod][pos] = (uint16_t)nb;
                    }
                    m += __popc(b);
                }
            }
            if (start + m > (uint32_t)kPool) overflow = true;
            if (overflow) {
                if (lane == 0) set_err(a, kPoolFull, e);
                return false;
            }
            if (lane == 0) {
                S.boff[prod][i] = (uint16_t)start;
                S.blen[prod][i] = (uint16_t)m;
                S.bump[prod] = start + m;
            }
            __syncwarp();
        }
        if (claimed_pass == 0) break;
    }
    // centroids (GetCentroids, DVCWeights.cxx:202-230): one lane per point, cells in order
    bool unowned = false;
    for (int p = lane; p < n; p += 32) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        int cnt = 0;
        for (int c = 0; c < a.ncell; c++) {
            if (S.owner[c] != p) continue;
            s0 = __dadd_rn(s0, S.cx[c % a.nx]);
            s1 = __dadd_rn(s1, S.cy[(c / a.nx) % a.ny]);
            if (DIM == 3) s2 = __dadd_rn(s2, S.cz[c / (a.nx * a.ny)]);
            cnt++;
        }
        if (cnt) {
            s0 = __ddiv_rn(s0, (double)cnt);
            s1 = __ddiv_rn(s1, (double)cnt);
            if (DIM == 3) s2 = __ddiv_rn(s2, (double)cnt);
        }
        S.cent[p][0] = s0;
        S.cent[p][1] = s1;
        S.cent[p][2] = s2;
        S.cnt[p] = (uint16_t)cnt;
    }
    for (int c = lane; c < a.ncell; c += 32)
        if (S.owner[c] == kNone) unowned = true;
    if (__any_sync(full, unowned)) {
        if (lane == 0) set_err(a, kUnowned, e);
        return false;
    }
    __syncwarp();
    return true;
}

template <int DIM>
__global__ void __launch_bounds__(32 * kWarps) k_dvc(DvcArgs a) {
    extern __shared__ unsigned char smem_raw[];
    DvcSmem& S = reinterpret_cast<DvcSmem*>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (e >= a.nel) return;
    const int32_t off = a.offsets[e];
    const int n = a.offsets[e + 1] - off;
    if (a.pc && lane == 0) {
        a.nsplit[e] = 0;
        a.ndel[e] = 0;
    }
    if (n == 0) return;
    if (n > kMaxPts || (a.pc && n + a.max_splits > kMaxPts)) {
        if (lane == 0) set_err(a, kTooMany, e);
        return;
    }
    // cell centres by the grid constructor's repeated additions (DVCWeights.cxx:557-575)
    if (lane == 0) {
        double X = __dsub_rn(-1.0, __ddiv_rn(a.dx, 2.0));
        for (int i = 0; i < a.nx; i++) S.cx[i] = X = __dadd_rn(X, a.dx);
        double Y = __dsub_rn(-1.0, __ddiv_rn(a.dy, 2.0));
        for (int j = 0; j < a.ny; j++) S.cy[j] = Y = __dadd_rn(Y, a.dy);
        double Z = __dsub_rn(-1.0, __ddiv_rn(a.dz, 2.0));
        for (int k = 0; k < a.nz; k++) S.cz[k] = Z = __dadd_rn(Z, a.dz);
    }
    for (int i = lane; i < n; i += 32) {
#pragma unroll
        for (int d = 0; d < 3; d++) S.xi[i][d] = d < DIM ? a.xi_s[(int64_t)d * a.np + off + i] : 0.0;
        S.list[i] = (int16_t)i;
    }
    __syncwarp();
    if (!dvc_warp<DIM>(a, S, n, e)) return;
    int m = n, nsplit = 0;
    if (a.pc) {
        // decisions (PCDVC.cxx:940-1013): lane 0
        if (lane == 0) {
            int maxD = a.max_deletions, maxS = a.max_splits;
            const int m0 = a.mat_s[off];
            for (int i = 0; i < n; i++)
                if (a.mat_s[off + i] != m0) {
                    if (!a.delete_if) maxD = 0;
                    if (!a.split_if) maxS = 0;
                    break;
                }
            int ns = 0, nd = 0;
            for (int i = 0; i < n; i++) {
                const double w = __dmul_rn((double)S.cnt[i], a.da);
                if (w > a.maxW) S.split[ns++] = (int16_t)i;
                if (w < a.minW) S.del[nd++] = (int16_t)i;
            }
            for (int x = 1; x < nd; x++)  // decreasing point index
                for (int y = x; y > 0 && a.perm[off + S.del[y - 1]] < a.perm[off + S.del[y]]; y--) {
                    const int16_t tmp = S.del[y];
                    S.del[y] = S.del[y - 1];
                    S.del[y - 1] = tmp;
                }
            if (maxD > n - 4) maxD = n / 2;
            nsplit = maxS > ns ? ns : maxS;
            const int ndel = maxD > nd ? nd : maxD;
            // new points: appended, at their parent's centroid
            for (int s = 0; s < nsplit; s++) {
                S.list[m] = (int16_t)(-1 - s);
                for (int d = 0; d < 3; d++) S.xi[m][d] = S.cent[S.split[s]][d];
                m++;
            }
            // deletions: the list's last entry takes the deleted entry's place
            for (int q = 0; q < ndel; q++) {
                int pos = 0;
                for (int k = 0; k < m; k++)
                    if (S.list[k] == S.del[q]) pos = k;
                S.list[pos] = S.list[m - 1];
                for (int d = 0; d < 3; d++) S.xi[pos][d] = S.xi[m - 1][d];
                m--;
                a.keep[off + S.del[q]] = 0;
            }
            a.nsplit[e] = nsplit;
            a.ndel[e] = ndel;
            S.bump[0] = (uint32_t)m;
            S.bump[1] = (uint32_t)nsplit;
        }
        __syncwarp();
        m = (int)S.bump[0];
        nsplit = (int)S.bump[1];
        if (m != n || nsplit) {
            if (m < 3) {  // the reference stops the run (PCDVC.cxx:1049)
                if (lane == 0) set_err(a, kTooFew, e);
                return;
            }
            if (!dvc_warp<DIM>(a, S, m, e)) return;
        }
    }
    // results of the final diagram
    for (int k = lane; k < m; k += 32) {
        const int src = S.list[k];
        const double w = __dmul_rn((double)S.cnt[k], a.da);
        if (src >= 0) {
            const int64_t i = off + src;
#pragma unroll
            for (int d = 0; d < DIM; d++) a.cent_out[(int64_t)d * a.np + i] = S.cent[k][d];
            a.w_out[i] = w;
        } else {
            const int s = -1 - src;
            const int64_t q = e * a.stride + s;
            a.new_parent[q] = off + S.split[s];
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                a.new_xi[q * DIM + d] = S.xi[k][d];
                a.new_cent[q * DIM + d] = S.cent[k][d];
            }
            a.new_w[q] = w;
        }
    }
}

// ---- rebuilding the point set after population control ------------------------------
__global__ void k_fill_u8(int64_t n, uint8_t v, uint8_t* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = v;
}

// sorted → point order: keep flags and integration points
__global__ void k_unsort(int64_t np, int dim, const int32_t* __restrict__ perm, const uint8_t* __restrict__ keep_s,
                         const double* __restrict__ cent_s, const double* __restrict__ w_s, int32_t* __restrict__ keep_p,
                         double* __restrict__ xi_p, double* __restrict__ w_p) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = perm[i];
        keep_p[p] = keep_s[i];
        w_p[p] = w_s[i];
        for (int d = 0; d < dim; d++) xi_p[(int64_t)p * dim + d] = cent_s[(int64_t)d * np + i];
    }
}

__global__ void k_compact(int64_t np, int dim, const int32_t* __restrict__ keep_p, const int32_t* __restrict__ newidx,
                          const double* __restrict__ coords, const int32_t* __restrict__ mat, const double* __restrict__ ps,
                          const double* __restrict__ xi_p, const double* __restrict__ w_p, double* __restrict__ coords2,
                          int32_t* __restrict__ mat2, double* __restrict__ ps2, double* __restrict__ xi2,
                          double* __restrict__ w2) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
        if (!keep_p[p]) continue;
        const int64_t q = newidx[p];
        for (int d = 0; d < dim; d++) {
            coords2[q * dim + d] = coords[p * dim + d];
            xi2[q * dim + d] = xi_p[p * dim + d];
        }
        mat2[q] = mat[p];
        ps2[q] = ps[p];
        w2[q] = w_p[p];
    }
}

// FeMesh_CoordLocalToGlobal (StgFEM/Discretisation/src/FeMesh.cxx:366-400) with the
// reference's rounding order: N_a by left-to-right products, x = Σ_a N_a x_a in node order
template <int DIM>
__device__ void local_to_global(const MeshK& mk, int64_t e, const double* xi, double* x) {
    const int i = (int)(e % mk.n[0]);
    const int64_t r = e / mk.n[0];
    const int j = (int)(r % mk.n[1]), k = (int)(r / mk.n[1]);
    for (int d = 0; d < DIM; d++) x[d] = 0.0;
#pragma unroll
    for (int a = 0; a < (1 << DIM); a++) {
        double N;
        if (DIM == 2) {
            N = __dmul_rn(__dmul_rn(0.25, __dadd_rn(1.0, (a & 1) ? xi[0] : -xi[0])),
                          __dadd_rn(1.0, (a & 2) ? xi[1] : -xi[1]));
        } else {
            N = __dmul_rn(__dmul_rn(__dmul_rn(0.125, __dadd_rn(1.0, (a & 1) ? xi[0] : -xi[0])),
                                    __dadd_rn(1.0, (a & 2) ? xi[1] : -xi[1])),
                          __dadd_rn(1.0, (a & 4) ? xi[2] : -xi[2]));
        }
        const int idx[3] = {i + (a & 1), j + ((a >> 1) & 1), k + ((a >> 2) & 1)};
        for (int d = 0; d < DIM; d++) x[d] = __dadd_rn(x[d], __dmul_rn(N, vert_coord_d(mk, d, idx[d])));
    }
}

template <int DIM>
__global__ void k_emit_new(MeshK mk, int64_t nel, int max_splits, int64_t base, const int32_t* __restrict__ nsplit,
                           const int32_t* __restrict__ newoff, const int32_t* __restrict__ new_parent,
                           const double* __restrict__ new_xi, const double* __restrict__ new_cent,
                           const double* __restrict__ new_w, const int32_t* __restrict__ perm,
                           const int32_t* __restrict__ mat, const double* __restrict__ ps, double* __restrict__ coords2,
                           int32_t* __restrict__ mat2, double* __restrict__ ps2, double* __restrict__ xi2,
                           double* __restrict__ w2) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
        for (int s = 0; s < nsplit[e]; s++) {
            const int64_t q = e * max_splits + s;
            const int64_t o = base + newoff[e] + s;
            const int32_t parent = perm[new_parent[q]];
            double x[3];
            local_to_global<DIM>(mk, e, new_xi + q * DIM, x);
            for (int d = 0; d < DIM; d++) {
                coords2[o * DIM + d] = x[d];
                xi2[o * DIM + d] = new_cent[q * DIM + d];
            }
            mat2[o] = mat[parent];
            ps2[o] = ps[parent];
            w2[o] = new_w[q];
        }
    }
}

// integration points (point order) → sorted arrays of the build
__global__ void k_apply_int(int64_t np, int dim, const int32_t* __restrict__ perm, const double* __restrict__ xi_p,
                            const double* __restrict__ w_p, double* __restrict__ xi_s, double* __restrict__ w_s) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = perm[i];
        w_s[i] = w_p[p];
        for (int d = 0; d < dim; d++) xi_s[(int64_t)d * np + i] = xi_p[(int64_t)p * dim + d];
    }
}

__global__ void k_copy_d(int64_t n, const double* __restrict__ a, double* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

const char* dvc_message(int code) {
    switch (code) {
        case kTooMany: return "more points in an element than the Voronoi kernel holds (254, less max_splits)";
        case kPoolFull: return "Voronoi boundary lists overflowed";
        case kPasses: return "Voronoi growth did not finish";
        case kUnowned: return "a Voronoi grid cell stayed unowned";
        case kTooFew: return "population control left fewer than 3 points in an element";
        default: return "Voronoi kernel error";
    }
}

}  // namespace

void exclusive_scan_i32(Handle& H, const int32_t* in, int32_t* out, int64_t n, DBuf& tmp, int32_t* total_host);

// DVC diagrams of every element of the located points; with `prm` also the population
// control and the rebuilt point set.  Leaves the integration points in H.xi_s / H.w_s.
int dvc_update(Handle& H, const gg_pcdvc_params* prm, gg_pcdvc_stats* stats) {
    const int dim = H.dim;
    const gg_weights& W = H.weights;
    const int nx = W.resolution[0], ny = W.resolution[1], nz = dim == 3 ? W.resolution[2] : 1;
    if (nx < 1 || ny < 1 || nz < 1 || nx > kAxis || ny > kAxis || nz > kAxis || nx * ny * nz > kMaxCells)
        return set_error(H, GG_ERR_INVALID, "DVC resolution: at most 64 per axis and 1024 cells per element");
    if (prm && (prm->inflow || prm->max_splits < 0 || prm->max_deletions < 0 || prm->max_splits >= kMaxPts))
        return set_error(H, GG_ERR_INVALID, "population control: Inflow is not provided; limits must be in range");
    cudaStream_t st = H.stream;
    const int64_t np = H.np, nel = H.nel;
    const int ms = prm ? std::max(prm->max_splits, 1) : 1;
    H.dvc_cent.ensure(sizeof(double) * np * dim);
    H.w_s.ensure(sizeof(double) * np);
    H.dvc_keep.ensure(np);
    H.dvc_err.ensure(sizeof(int32_t) * 2);
    if (prm) {
        H.dvc_nsplit.ensure(sizeof(int32_t) * (nel + 1));
        H.dvc_ndel.ensure(sizeof(int32_t) * (nel + 1));
        H.dvc_parent.ensure(sizeof(int32_t) * nel * ms);
        H.dvc_new.ensure(sizeof(double) * nel * ms * (2 * dim + 1));
    }
    // the diagrams grow from the material points: keep their ξ apart from the integration
    // points that replace xi_s
    H.xi_pts.ensure(sizeof(double) * np * dim);
    if (!H.dvc_valid)
        GG_CUDA(cudaMemcpyAsync(H.xi_pts.p, H.xi_s.p, sizeof(double) * np * dim, cudaMemcpyDeviceToDevice, st));
    GG_CUDA(cudaMemsetAsync(H.dvc_err.p, 0, sizeof(int32_t) * 2, st));
    k_fill_u8<<<grid_for(np, 256), 256, 0, st>>>(np, 1, H.dvc_keep.as<uint8_t>());
    DvcArgs a{};
    a.dim = dim;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.ncell = nx * ny * nz;
    a.dx = (1.0 - -1.0) / nx;
    a.dy = (1.0 - -1.0) / ny;
    a.dz = dim == 3 ? (1.0 - -1.0) / nz : 1.0;
    a.da = dim == 3 ? a.dx * a.dy * a.dz : a.dx * a.dy;
    a.nel = nel;
    a.np = np;
    a.offsets = H.offsets.as<int32_t>();
    a.xi_s = H.xi_pts.as<double>();
    a.mat_s = H.mat_s.as<int32_t>();
    a.perm = H.perm.as<int32_t>();
    a.cent_out = H.dvc_cent.as<double>();
    a.w_out = H.w_s.as<double>();
    a.keep = H.dvc_keep.as<uint8_t>();
    a.err = H.dvc_err.as<int32_t>();
    if (prm) {
        const double vol = dim == 3 ? 8.0 : 4.0;
        a.pc = 1;
        a.maxW = prm->upper_t * vol / 100.0;
        a.minW = prm->lower_t * vol / 100.0;
        a.max_splits = prm->max_splits;
        a.max_deletions = prm->max_deletions;
        a.split_if = prm->split_in_interface_cells;
        a.delete_if = prm->delete_in_interface_cells;
        a.stride = ms;
        a.new_parent = H.dvc_parent.as<int32_t>();
        double* nb = H.dvc_new.as<double>();
        a.new_xi = nb;
        a.new_cent = nb + nel * ms * dim;
        a.new_w = nb + 2 * nel * ms * dim;
        a.nsplit = H.dvc_nsplit.as<int32_t>();
        a.ndel = H.dvc_ndel.as<int32_t>();
    }
    const size_t smem = sizeof(DvcSmem) * kWarps;
    const int blocks = (int)((nel + kWarps - 1) / kWarps);
    if (dim == 2) {
        GG_CUDA(cudaFuncSetAttribute(k_dvc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_dvc<2><<<blocks, 32 * kWarps, smem, st>>>(a);
    } else {
        GG_CUDA(cudaFuncSetAttribute(k_dvc<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_dvc<3><<<blocks, 32 * kWarps, smem, st>>>(a);
    }
    GG_CUDA(cudaGetLastError());
    int32_t err[2] = {0, 0};
    GG_CUDA(cudaMemcpyAsync(err, H.dvc_err.p, sizeof err, cudaMemcpyDeviceToHost, st));
    GG_CUDA(cudaStreamSynchronize(st));
    if (err[0])
        return set_error(H, GG_ERR_INVALID, std::string(dvc_message(err[0])) + " (element " + std::to_string(err[1]) + ")");
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->points_before = np;
        stats->points_after = np;
    }
    if (!prm) {
        k_copy_d<<<grid_for(np * dim, 256), 256, 0, st>>>(np * dim, H.dvc_cent.as<double>(), H.xi_s.as<double>());
        GG_CUDA(cudaGetLastError());
        H.dvc_valid = true;
        return GG_OK;
    }
    // totals of splits and deletions
    int32_t nsplit_tot = 0, ndel_tot = 0;
    H.dvc_scan.ensure(sizeof(int32_t) * (nel + 1));
    exclusive_scan_i32(H, H.dvc_nsplit.as<int32_t>(), H.dvc_scan.as<int32_t>(), nel, H.scan_tmp, &nsplit_tot);
    H.dvc_scan2.ensure(sizeof(int32_t) * (nel + 1));
    exclusive_scan_i32(H, H.dvc_ndel.as<int32_t>(), H.dvc_scan2.as<int32_t>(), nel, H.scan_tmp, &ndel_tot);
    if (stats) {
        stats->splits = nsplit_tot;
        stats->deletions = ndel_tot;
        stats->points_after = np + nsplit_tot - ndel_tot;
    }
    if (nsplit_tot == 0 && ndel_tot == 0) {
        k_copy_d<<<grid_for(np * dim, 256), 256, 0, st>>>(np * dim, H.dvc_cent.as<double>(), H.xi_s.as<double>());
        GG_CUDA(cudaGetLastError());
        H.dvc_valid = true;
        return GG_OK;
    }
    // point order: keep flags, integration points
    DBuf keep_p, newidx, xi_p, w_p;
    keep_p.ensure(sizeof(int32_t) * np);
    newidx.ensure(sizeof(int32_t) * (np + 1));
    xi_p.ensure(sizeof(double) * np * dim);
    w_p.ensure(sizeof(double) * np);
    k_unsort<<<grid_for(np, 256), 256, 0, st>>>(np, dim, H.perm.as<int32_t>(), H.dvc_keep.as<uint8_t>(),
                                                 H.dvc_cent.as<double>(), H.w_s.as<double>(), keep_p.as<int32_t>(),
                                                 xi_p.as<double>(), w_p.as<double>());
    int32_t nsurv = 0;
    exclusive_scan_i32(H, keep_p.as<int32_t>(), newidx.as<int32_t>(), np, H.scan_tmp, &nsurv);
    const int64_t np2 = (int64_t)nsurv + nsplit_tot;
    DBuf coords2, mat2, ps2, xi2, w2;
    coords2.ensure(sizeof(double) * np2 * dim);
    mat2.ensure(sizeof(int32_t) * np2);
    ps2.ensure(sizeof(double) * np2);
    xi2.ensure(sizeof(double) * np2 * dim);
    w2.ensure(sizeof(double) * np2);
    k_compact<<<grid_for(np, 256), 256, 0, st>>>(np, dim, keep_p.as<int32_t>(), newidx.as<int32_t>(),
                                                  H.coords.as<double>(), H.mat_in.as<int32_t>(), H.ps_in.as<double>(),
                                                  xi_p.as<double>(), w_p.as<double>(), coords2.as<double>(),
                                                  mat2.as<int32_t>(), ps2.as<double>(), xi2.as<double>(), w2.as<double>());
    double* nb = H.dvc_new.as<double>();
    if (dim == 2)
        k_emit_new<2><<<grid_for(nel, 256), 256, 0, st>>>(
            H.mk, nel, ms, nsurv, H.dvc_nsplit.as<int32_t>(), H.dvc_scan.as<int32_t>(), H.dvc_parent.as<int32_t>(), nb,
            nb + nel * ms * dim, nb + 2 * nel * ms * dim, H.perm.as<int32_t>(), H.mat_in.as<int32_t>(),
            H.ps_in.as<double>(), coords2.as<double>(), mat2.as<int32_t>(), ps2.as<double>(), xi2.as<double>(),
            w2.as<double>());
    else
        k_emit_new<3><<<grid_for(nel, 256), 256, 0, st>>>(
            H.mk, nel, ms, nsurv, H.dvc_nsplit.as<int32_t>(), H.dvc_scan.as<int32_t>(), H.dvc_parent.as<int32_t>(), nb,
            nb + nel * ms * dim, nb + 2 * nel * ms * dim, H.perm.as<int32_t>(), H.mat_in.as<int32_t>(),
            H.ps_in.as<double>(), coords2.as<double>(), mat2.as<int32_t>(), ps2.as<double>(), xi2.as<double>(),
            w2.as<double>());
    GG_CUDA(cudaGetLastError());
    GG_CUDA(cudaStreamSynchronize(st));
    // the new point set replaces the old one; per-point work arrays follow its size
    std::swap(H.coords.p, coords2.p);
    std::swap(H.coords.bytes, coords2.bytes);
    std::swap(H.mat_in.p, mat2.p);
    std::swap(H.mat_in.bytes, mat2.bytes);
    std::swap(H.ps_in.p, ps2.p);
    std::swap(H.ps_in.bytes, ps2.bytes);
    H.np = np2;
    for (DBuf* b : {&H.cell, &H.perm, &H.cell_s, &H.mat_s}) b->ensure(sizeof(int32_t) * np2);
    for (DBuf* b : {&H.ps_s, &H.eta_s, &H.incr_s, &H.w_s}) b->ensure(sizeof(double) * np2);
    H.xi_s.ensure(sizeof(double) * np2 * dim);
    H.yld_s.ensure(np2);
    const int64_t outside = locate_and_sort(H);
    H.np_in = np2 - outside;
    if (outside) return set_error(H, GG_ERR_OUT_OF_DOMAIN, "a new point left the mesh");
    H.xi_pts.ensure(sizeof(double) * np2 * dim);
    GG_CUDA(cudaMemcpyAsync(H.xi_pts.p, H.xi_s.p, sizeof(double) * np2 * dim, cudaMemcpyDeviceToDevice, st));
    k_apply_int<<<grid_for(np2, 256), 256, 0, st>>>(np2, dim, H.perm.as<int32_t>(), xi2.as<double>(), w2.as<double>(),
                                                    H.xi_s.as<double>(), H.w_s.as<double>());
    GG_CUDA(cudaGetLastError());
    GG_CUDA(cudaStreamSynchronize(st));
    H.dvc_valid = true;
    return GG_OK;
}

}  // namespace gg
