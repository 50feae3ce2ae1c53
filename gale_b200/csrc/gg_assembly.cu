// gg_assembly.cu -- per-point viscosity and PIC quadrature moments on sm_100a.
//
// Replaces, for the Q1-P0 Stokes SLE, the per-element loops of
//   _ConstitutiveMatrixCartesian_AssembleElement (Underworld/Rheology/src/
//       ConstitutiveMatrixCartesian.cxx:206-487) and the rheology chain it runs per point
//       (Rheology_Register_RunRheologies, Rheology_Register.cxx:70-86),
//   _BuoyancyForceTerm_AssembleElement (PICellerator/Utils/src/BuoyancyForceTerm.cxx:414-530),
//   _ThermalBuoyancyForceTerm_AssembleElement (StgFEM/Assembly/src/
//       ThermalBuoyancyForceTerm.cxx:180-235),
//   _UzawaPreconditionerTerm_AssembleElement (StgFEM/SLE/ProvidedSystems/StokesFlow/src/
//       UzawaPreconditionerTerm.cxx:156-239).
//
// On an axis-aligned element B is polynomial in ξ, so K_e = Σ_p c_p Bᵀ D0 B with
// c_p = w_p detJ η_p is fixed by the moments M_m(e) = Σ_p c_p m(ξ_p) of the monomials
// m ∈ {ξ^a η^b ζ^c} that Bᵀ D0 B contains (6 in 2D, 23 in 3D).  One pass over the
// points (sorted by element, in reference order) produces them; the K apply then never
// touches a point again.
//
// Kernel shape: a CTA owns 128 consecutive elements and walks their contiguous point
// range in chunks of 512.  Phase 1 (one thread per point, coalesced loads): rheology,
// c_p, force weights → shared memory.  Phase 2 (one thread per element): sequential
// sums in point order, i.e. the reference's summation order.  The element's corner terms
// of the K diagonal and of the force go to per-element buffers; k_gather_corners sums
// them per node in a fixed element order, so a build gives the same bits on every run.
#include <map>
#include <set>
#include <condition_variable>
#include <mutex>
#include <tuple>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"

namespace gg {

namespace {

// CTA shapes (elements per CTA = threads, points per shared-memory chunk) the autotuner
// chooses from; the sums per element run in point order whatever the shape, so every
// shape gives the same moments.
struct BuildShape {
    int epc, chunk;
};
constexpr BuildShape kShapes[] = {{64, 256}, {128, 256}, {128, 512}, {256, 512}};
constexpr int kNumShapes = 4;

template <typename R> __device__ __forceinline__ R r_exp(R x);
template <> __device__ __forceinline__ double r_exp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float r_exp<float>(float x) { return expf(x); }
template <typename R> __device__ __forceinline__ R r_sqrt(R x);
template <> __device__ __forceinline__ double r_sqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float r_sqrt<float>(float x) { return sqrtf(x); }

// Q1 shape functions at ξ, node order of BilinearElementType/TrilinearElementType.
template <int DIM, typename R>
__device__ __forceinline__ void shape(const R* xi, R* N) {
#pragma unroll
    for (int a = 0; a < (1 << DIM); a++) {
        R v = (DIM == 2) ? R(0.25) : R(0.125);
#pragma unroll
        for (int d = 0; d < DIM; d++) v *= (R(1) + ((a >> d) & 1 ? xi[d] : -xi[d]));
        N[a] = v;
    }
}

// SymmetricTensor_2ndInvariant (StgDomain/Geometry/src/TensorMath.cxx:431-460).
template <int DIM, typename R>
__device__ __forceinline__ R second_invariant(const R* t) {
    if (DIM == 2) return r_sqrt<R>(R(0.5) * (t[0] * t[0] + t[1] * t[1]) + t[2] * t[2]);
    return r_sqrt<R>(R(0.5) * (t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) + t[3] * t[3] +
                     t[4] * t[4] + t[5] * t[5]);
}

struct PointOut {
    double eta, incr;
    uint8_t yielded;
};

// Rheology chain of one material point (RheologyMaterial_RunRheologies).
template <int DIM, typename R>
__device__ PointOut run_rheologies(const MeshK& mk, const gg_material& m, const int* ijk,
                                   int64_t e, const R* xi, const double* __restrict__ T,
                                   const double* __restrict__ pu, const double* __restrict__ pp,
                                   double ep_in, int prev) {
    R eta = R(0);
    R ep = (R)ep_in;
    PointOut out{0.0, 0.0, 0};
    R Tp = R(0);
    bool haveT = false;
    for (int ri = 0; ri < m.n_rheologies; ri++) {
        const gg_rheology& r = m.rheology[ri];
        const int kind = r.kind;
        if (kind == GG_RHEO_MATERIAL_VISCOSITY) {  // MaterialViscosity.cxx:139
            eta = (R)r.eta0;
        } else if (kind == GG_RHEO_ARRHENIUS || kind == GG_RHEO_FRANK_KAMENETSKII) {
            if (!haveT) {
                if (T) {
                    R N[1 << DIM];
                    shape<DIM, R>(xi, N);
                    Tp = R(0);
#pragma unroll
                    for (int a = 0; a < (1 << DIM); a++) Tp += (R)T[elem_node<DIM>(mk, ijk, a)] * N[a];
                }
                haveT = true;
            }
            if (kind == GG_RHEO_FRANK_KAMENETSKII) {  // FrankKamenetskii.cxx:156-160
                eta = (R)r.eta0 * r_exp<R>(-(R)r.theta * Tp);
            } else if (r.activation_volume > (0.0 + 1e-12)) {  // Arrhenius.cxx:200-214
                const R y = (R)(mk.min[1] + (ijk[1] + 0.5) * mk.h[1]) + xi[1] * (R)(0.5 * mk.h[1]);
                const R depth = (R)mk.max[1] - y;
                eta = (R)r.eta0 * r_exp<R>(((R)r.activation_energy + (R)r.activation_volume * depth) /
                                           (Tp + (R)r.reference_temp));
            } else {
                eta = (R)r.eta0 * r_exp<R>((R)r.activation_energy / (Tp + (R)r.reference_temp));
            }
        } else if (kind == GG_RHEO_VON_MISES || kind == GG_RHEO_DRUCKER_PRAGER ||
                   kind == GG_RHEO_BYERLEE) {
            // _YieldRheology_ModifyConstitutiveMatrix (YieldRheology.cxx:190-228)
            if (!prev) continue;
            // strain rate at ξ from the previous velocity: ε̇ = sym(∇u)
            R g[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
            for (int a = 0; a < (1 << DIM); a++) {
                const int64_t n = elem_node<DIM>(mk, ijk, a);
                R dN[3];
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    R v = (R)mk.kappa[d] * (((a >> d) & 1) ? R(1) : R(-1));
#pragma unroll
                    for (int o = 0; o < DIM; o++)
                        if (o != d) v *= (R(1) + (((a >> o) & 1) ? xi[o] : -xi[o]));
                    dN[d] = v;
                }
#pragma unroll
                for (int c = 0; c < DIM; c++) {
                    const R uc = (R)pu[(int64_t)c * mk.nnode + n];
#pragma unroll
                    for (int d = 0; d < DIM; d++) g[c][d] += dN[d] * uc;
                }
            }
            R sr[6], st[6];
            if (DIM == 2) {
                sr[0] = g[0][0]; sr[1] = g[1][1]; sr[2] = R(0.5) * (g[0][1] + g[1][0]);
            } else {
                sr[0] = g[0][0]; sr[1] = g[1][1]; sr[2] = g[2][2];
                sr[3] = R(0.5) * (g[0][1] + g[1][0]);
                sr[4] = R(0.5) * (g[0][2] + g[2][0]);
                sr[5] = R(0.5) * (g[1][2] + g[2][1]);
            }
            const int ns = DIM == 2 ? 3 : 6;
            R trs = R(0), trsr = R(0);
            for (int k = 0; k < ns; k++) st[k] = R(2) * eta * sr[k];  // isotropic D·ε̇
            for (int k = 0; k < DIM; k++) { trs += st[k]; trsr += sr[k]; }
            for (int k = 0; k < DIM; k++) { sr[k] -= trsr / R(DIM); st[k] -= trs / R(DIM); }
            const R sr_ii = second_invariant<DIM, R>(sr);
            const R ind = second_invariant<DIM, R>(st);  // _VonMises_GetYieldIndicator
            // StrainWeakening_CalcRatio (StrainWeakening.cxx:497-519)
            R ratio = R(0);
            const bool sw = m.has_strain_weakening && r.strain_weakening;
            if (sw) {
                if (ep < R(0)) ep = R(0);
                ratio = (ep - (R)m.strain_weakening.initial_softening_strain) /
                        ((R)m.strain_weakening.final_softening_strain -
                         (R)m.strain_weakening.initial_softening_strain);
                if (ratio > R(1)) ratio = R(1);
                if (ratio < R(0)) ratio = R(0);
            }
            R crit;
            if (kind == GG_RHEO_VON_MISES) {  // VonMises.cxx:183-204
                crit = (R)r.cohesion * (R(1) - ratio) + (R)r.cohesion_after_softening * ratio;
            } else if (kind == GG_RHEO_DRUCKER_PRAGER) {  // DruckerPrager.cxx:296-412
                const R pressure = pp ? (R)pp[e] : R(0);
                // elements along a flagged wall take the boundary strength (:341-361)
                const int bw = r.boundary_walls;
                const bool inb = ((bw & 1) && ijk[0] == 0) || ((bw & 2) && ijk[0] == mk.n[0] - 1) ||
                                 ((bw & 4) && ijk[1] == 0) || ((bw & 8) && ijk[1] == mk.n[1] - 1) ||
                                 (DIM == 3 && (((bw & 16) && ijk[2] == 0) || ((bw & 32) && ijk[2] == mk.n[2] - 1)));
                const R mu = inb ? (R)r.boundary_friction_coefficient * (R(1) - ratio) +
                                       (R)r.boundary_friction_coefficient_after_softening * ratio
                                 : (R)r.friction_coefficient * (R(1) - ratio) +
                                       (R)r.friction_coefficient_after_softening * ratio;
                const R C = inb ? (R)r.boundary_cohesion * (R(1) - ratio) + (R)r.boundary_cohesion_after_softening * ratio
                                : (R)r.cohesion * (R(1) - ratio) + (R)r.cohesion_after_softening * ratio;
                R factor, fs;
                if (DIM == 2) {
                    factor = R(1) / r_sqrt<R>(R(1) + mu * mu);
                    fs = mu * pressure * factor + C * factor;
                } else {
                    const R cphi = R(1) / r_sqrt<R>(R(1) + mu * mu), sphi = mu * cphi;
                    factor = R(2) * cphi / (r_sqrt<R>(R(3)) * (R(3) - sphi));
                    fs = mu * factor * pressure + C * R(3) * factor;
                }
                R mys = (R)r.minimum_yield_stress;
                if (mys == R(0)) mys = C;
                if (fs < mys * factor) fs = mys * factor;
                crit = fs;
            } else {  // Byerlee.cxx:163-187
                const R y = (R)(mk.min[1] + (ijk[1] + 0.5) * mk.h[1]) + xi[1] * (R)(0.5 * mk.h[1]);
                crit = (R)r.cohesion + (R)r.depth_coefficient * ((R)mk.max[1] - y);
            }
            if (sw) {  // _StrainWeakening_CalcIncrementIsotropic (StrainWeakening.cxx:470-495)
                R beta = R(1) - crit / ind;
                if (beta < R(0)) beta = R(0);
                out.incr = (double)((crit / eta) *
                                    (beta / (R(1) - beta) - (R)m.strain_weakening.healing_rate * ep));
            }
            if (crit < ind) {
                out.yielded = 1;
                if (kind == GG_RHEO_DRUCKER_PRAGER) {  // DruckerPrager.cxx:414-446
                    R v = (r.max_strain_rate > 0 && sr_ii > (R)r.max_strain_rate)
                              ? crit / (R(2) * (R)r.max_strain_rate)
                              : crit / (R(2) * sr_ii);
                    if (v < (R)r.minimum_viscosity) v = (R)r.minimum_viscosity;
                    eta = v;
                } else if (r.strain_rate_softening) {  // VonMises.cxx:258-263
                    eta = R(2) * crit * crit * eta / (crit * crit + ind * ind);
                } else {  // VonMises.cxx:264-271
                    const R beta = R(1) - crit / ind;
                    R corr = -eta * beta;
                    if ((eta + corr) < (R)r.minimum_viscosity) corr = (R)r.minimum_viscosity - eta;
                    eta += corr;
                }
            }
        }
    }
    out.eta = (double)eta;
    return out;
}

template <int DIM, typename R, int kElemPerCta, int kChunk>
__global__ void __launch_bounds__(kElemPerCta)
k_build_moments(MeshK mk, int64_t nel, const int32_t* __restrict__ offsets,
                const double* __restrict__ xi_s, int64_t np_s, const int32_t* __restrict__ mat_s,
                const double* __restrict__ ps_s, const double* __restrict__ T,
                const double* __restrict__ pu, const double* __restrict__ pp, int prev,
                double gravity, double g0, double g1, double g2, double rayleigh, int want_force,
                R* __restrict__ mom, R* __restrict__ kcorner, double* __restrict__ sdiag,
                double* __restrict__ fcorner, double* __restrict__ eta_s, double* __restrict__ incr_s,
                uint8_t* __restrict__ yld_s, int32_t* __restrict__ flag,
                const gg_material* __restrict__ materials, const double* __restrict__ w_s) {
    constexpr int NM = n_moments<DIM>();
    constexpr int NEN = 1 << DIM;
    __shared__ R s_c[kChunk];
    __shared__ R s_xi[DIM][kChunk];
    __shared__ double s_phi[kChunk];
    __shared__ double s_psi[kChunk];

    const int64_t e0 = (int64_t)blockIdx.x * kElemPerCta;
    if (e0 >= nel) return;
    const int64_t e1 = min(nel, e0 + kElemPerCta);
    const int64_t e = e0 + threadIdx.x;
    const bool own = e < e1;
    const int32_t pbeg = offsets[e0], pend = offsets[e1];
    const int32_t my_b = own ? offsets[e] : 0, my_e = own ? offsets[e + 1] : 0;
    const double wscale = (double)(1 << DIM);

    R acc[NM];
#pragma unroll
    for (int m = 0; m < NM; m++) acc[m] = R(0);
    double F[NEN], Psi[NEN];
#pragma unroll
    for (int a = 0; a < NEN; a++) { F[a] = 0.0; Psi[a] = 0.0; }

    for (int32_t cs = pbeg; cs < pend; cs += kChunk) {
        const int32_t ce = min(pend, cs + kChunk);
        // ---- phase 1: one thread per point
        for (int32_t i = cs + threadIdx.x; i < ce; i += blockDim.x) {
            // element of sorted point i: binary search in this CTA's offsets
            int lo = 0, hi = (int)(e1 - e0) - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (offsets[e0 + mid] <= i) lo = mid; else hi = mid - 1;
            }
            const int64_t pe = e0 + lo;
            int ijk[3];
            elem_ijk(mk, pe, ijk);
            R xi[3] = {R(0), R(0), R(0)};
#pragma unroll
            for (int d = 0; d < DIM; d++) xi[d] = (R)xi_s[(int64_t)d * np_s + i];
            const int mi = mat_s[i];
            const gg_material& m = materials[mi];
            PointOut po = run_rheologies<DIM, R>(mk, m, ijk, pe, xi, T, pu, pp, ps_s[i], prev);
            const int32_t cnt = offsets[pe + 1] - offsets[pe];
            // per-point weight (DVCWeights) or _ConstantWeights_Calculate
            const double w = w_s ? w_s[i] : wscale / (double)cnt;
            s_c[i - cs] = (R)(w * mk.detJ) * (R)po.eta;
#pragma unroll
            for (int d = 0; d < DIM; d++) s_xi[d][i - cs] = xi[d];
            if (want_force) {
                double Tp = 0.0;
                if (T && (rayleigh != 0.0 || m.alpha != 0.0)) {
                    double xd[3] = {xi_s[i], xi_s[np_s + i], DIM == 3 ? xi_s[2 * np_s + i] : 0.0};
                    double N[NEN];
                    shape<DIM, double>(xd, N);
#pragma unroll
                    for (int a = 0; a < NEN; a++) Tp += T[elem_node<DIM>(mk, ijk, a)] * N[a];
                }
                const double rho = m.density * (1.0 - m.alpha * Tp);
                s_phi[i - cs] = mk.detJ * w * rho * gravity;
                s_psi[i - cs] = mk.detJ * w * (rayleigh * Tp);
            }
            if (eta_s) {
                eta_s[i] = po.eta;
                incr_s[i] = po.incr;
                yld_s[i] = po.yielded;
            }
        }
        __syncthreads();
        // ---- phase 2: one thread per element, points in reference order
        if (own) {
            const int32_t b = max(my_b, cs), en = min(my_e, ce);
            for (int32_t i = b; i < en; i++) {
                const int k = i - cs;
                const R c = s_c[k];
                R px[3], py[3], pz[3];
                px[0] = R(1); px[1] = s_xi[0][k]; px[2] = px[1] * px[1];
                py[0] = R(1); py[1] = s_xi[1][k]; py[2] = py[1] * py[1];
                pz[0] = R(1); pz[1] = DIM == 3 ? s_xi[DIM - 1][k] : R(0); pz[2] = pz[1] * pz[1];
#pragma unroll
                for (int cc = 0; cc < (DIM == 3 ? 3 : 1); cc++)
#pragma unroll
                    for (int bb = 0; bb < 3; bb++)
#pragma unroll
                        for (int aa = 0; aa < 3; aa++) {
                            constexpr int dummy = 0;
                            (void)dummy;
                            const int slot = mom_slot<DIM>(aa, bb, cc);
                            if (slot >= 0) acc[slot] += c * (px[aa] * py[bb] * pz[cc]);
                        }
                if (want_force) {
                    double xd[3] = {(double)s_xi[0][k], (double)s_xi[1][k],
                                    DIM == 3 ? (double)s_xi[DIM - 1][k] : 0.0};
                    double N[NEN];
                    shape<DIM, double>(xd, N);
                    const double phi = s_phi[k], psi = s_psi[k];
#pragma unroll
                    for (int a = 0; a < NEN; a++) { F[a] += phi * N[a]; Psi[a] += psi * N[a]; }
                }
            }
        }
        __syncthreads();
    }
    if (!own) return;
    if (my_e == my_b) atomicAdd(flag, 1);  // empty element
#pragma unroll
    for (int m = 0; m < NM; m++) mom[(int64_t)m * nel + e] = acc[m];

    // element diagonal of K from the moments:
    // K[(a,c),(a,c)] = Σ_p c_p [ Σ_d (∂N_a/∂x_d)² + (∂N_a/∂x_c)² ]
    int ijk[3];
    elem_ijk(mk, e, ijk);
    double sd = 0.0;
#pragma unroll
    for (int a = 0; a < NEN; a++) {
        double S[3];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            // Σ_p c_p Π_{o≠d} (1 + s_o ξ_o)²,  (1+sξ)² = 1 + 2sξ + ξ²
            double v = 0.0;
#pragma unroll
            for (int k0 = 0; k0 < 3; k0++)
#pragma unroll
                for (int k1 = 0; k1 < 3; k1++)
#pragma unroll
                    for (int k2 = 0; k2 < 3; k2++) {
                        int ex[3] = {k0, k1, k2};
                        bool ok = true;
                        double coef = 1.0;
#pragma unroll
                        for (int o = 0; o < 3; o++) {
                            if (o >= DIM || o == d) { if (ex[o] != 0) ok = false; continue; }
                            const double s = ((a >> o) & 1) ? 1.0 : -1.0;
                            coef *= ex[o] == 1 ? 2.0 * s : 1.0;
                        }
                        if (!ok) continue;
                        const int slot = mom_slot<DIM>(k0, k1, k2);
                        v += coef * (double)acc[slot];
                    }
            S[d] = v * mk.kappa[d] * mk.kappa[d];
        }
        double tot = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) tot += S[d];
#pragma unroll
        for (int c = 0; c < DIM; c++) {
            const double dg = tot + S[c];
            kcorner[(int64_t)(a * DIM + c) * nel + e] = (R)dg;
            // Ĝ_e = Σ G_e² / K_e diagonal, over every dof (UzawaPreconditionerTerm.cxx:199-215)
            sd += mk.Ge[a][c] * (mk.Ge[a][c] / dg);
        }
        if (want_force) {
            fcorner[(int64_t)a * nel + e] = F[a];
            fcorner[(int64_t)(NEN + a) * nel + e] = Psi[a];
        }
    }
    if (sdiag) sdiag[e] = sd;
}

// Node sums of the element corner terms in a fixed element order (corner a' = 0 … 2^dim−1
// of the node in its adjacent elements), so the assembled diagonal and force vector are
// the same bits on every run: kdiag[c][n] = Σ_e K_e[(a',c),(a',c)],
// f[c][n] = Σ_e (g_c F_e[a'] + [c = y] Ψ_e[a']).
template <int DIM, typename R>
__global__ void k_gather_corners(MeshK mk, const R* __restrict__ kcorner, const double* __restrict__ fcorner,
                                 double g0, double g1, double g2, R* __restrict__ kdiag, double* __restrict__ f) {
    constexpr int NEN = 1 << DIM;
    const int64_t nnode = mk.nnode, nel = mk.nel;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nnode; n += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(n % mk.nn[0]);
        const int j = (int)((n / mk.nn[0]) % mk.nn[1]);
        const int k = DIM == 3 ? (int)(n / ((int64_t)mk.nn[0] * mk.nn[1])) : 0;
        R kd[DIM];
        double fv[DIM];
#pragma unroll
        for (int c = 0; c < DIM; c++) { kd[c] = R(0); fv[c] = 0.0; }
#pragma unroll
        for (int a = 0; a < NEN; a++) {
            const int ei = i - (a & 1), ej = j - ((a >> 1) & 1), ek = DIM == 3 ? k - ((a >> 2) & 1) : 0;
            if (ei < 0 || ej < 0 || ek < 0 || ei >= mk.n[0] || ej >= mk.n[1] || (DIM == 3 && ek >= mk.n[2])) continue;
            const int64_t e = ei + (int64_t)mk.n[0] * (ej + (int64_t)mk.n[1] * ek);
#pragma unroll
            for (int c = 0; c < DIM; c++) kd[c] += kcorner[(int64_t)(a * DIM + c) * nel + e];
            if (f) {
                const double Fa = fcorner[(int64_t)a * nel + e], Pa = fcorner[(int64_t)(NEN + a) * nel + e];
#pragma unroll
                for (int c = 0; c < DIM; c++) {
                    double v = (c == 0 ? g0 : (c == 1 ? g1 : g2)) * Fa;
                    if (c == 1) v += Pa;
                    fv[c] += v;
                }
            }
        }
#pragma unroll
        for (int c = 0; c < DIM; c++) {
            kdiag[(int64_t)c * nnode + n] = kd[c];
            if (f) f[(int64_t)c * nnode + n] = fv[c];
        }
    }
}

}  // namespace

// The material table lives in a per-handle device buffer, so concurrent handles (threads,
// streams) never share it.
void upload_materials(Handle& H) {
    H.d_materials.ensure(sizeof(gg_material) * GG_MAX_MATERIALS);
    H.h_materials.assign(H.materials.begin(), H.materials.end());
    GG_CUDA(cudaMemcpyAsync(H.d_materials.p, H.h_materials.data(), sizeof(gg_material) * H.h_materials.size(),
                            cudaMemcpyHostToDevice, H.stream));
}

template <int DIM, typename R, int EPC, int CH>
static void launch_shape(Handle& H, int prev, const double* pu, const double* pp, R* mom, R* kdiag, double* sdiag,
                         double* f, bool outputs) {
    const int64_t nel = H.nel;
    const int grid = (int)((nel + EPC - 1) / EPC);
    const double* T = H.has_T ? H.T.as<double>() : nullptr;
    double g[3] = {H.force.g_hat[0], H.force.g_hat[1], H.force.g_hat[2]};
    k_build_moments<DIM, R, EPC, CH><<<grid, EPC, 0, H.stream>>>(
        H.mk, nel, H.offsets.as<int32_t>(), H.xi_s.as<double>(), H.np_in, H.mat_s.as<int32_t>(),
        H.ps_s.as<double>(), T, pu, pp, prev, H.force.gravity, g[0], g[1], g[2], H.force.rayleigh,
        f ? 1 : 0, mom, reinterpret_cast<R*>(H.kcorner.p), sdiag, f ? H.fcorner.as<double>() : nullptr,
        outputs ? H.eta_s.as<double>() : nullptr,
        H.incr_s.as<double>(), H.yld_s.as<uint8_t>(), H.flag.as<int32_t>(), H.d_materials.as<gg_material>(),
        H.weights.mode == GG_WEIGHTS_DVC && H.dvc_valid ? H.w_s.as<double>() : nullptr);
    GG_CUDA(cudaGetLastError());
}

// kdiag (and f) from the corner terms of the last build launch
template <int DIM, typename R>
static void gather_corners(Handle& H, R* kdiag, double* f) {
    double g[3] = {H.force.g_hat[0], H.force.g_hat[1], H.force.g_hat[2]};
    const double* fc = f ? H.fcorner.as<double>() : nullptr;
    k_gather_corners<DIM, R><<<grid_for(H.nnode, 256), 256, 0, H.stream>>>(
        H.mk, reinterpret_cast<const R*>(H.kcorner.p), fc, g[0], g[1], g[2], kdiag, f);
    GG_CUDA(cudaGetLastError());
}

template <int DIM, typename R>
static void launch_build_shape(int shape, Handle& H, int prev, const double* pu, const double* pp, R* mom, R* kdiag,
                               double* sdiag, double* f, bool outputs) {
    switch (shape) {
        case 0: launch_shape<DIM, R, 64, 256>(H, prev, pu, pp, mom, kdiag, sdiag, f, outputs); break;
        case 1: launch_shape<DIM, R, 128, 256>(H, prev, pu, pp, mom, kdiag, sdiag, f, outputs); break;
        case 2: launch_shape<DIM, R, 128, 512>(H, prev, pu, pp, mom, kdiag, sdiag, f, outputs); break;
        default: launch_shape<DIM, R, 256, 512>(H, prev, pu, pp, mom, kdiag, sdiag, f, outputs); break;
    }
}

// Autotuner: the first build of a (device, dim, precision, points-per-element class) times
// every CTA shape twice on the real inputs (each trial overwrites every output) and keeps
// the fastest for the rest of the process.  One thread tunes a key while the builds of
// other threads with the same key wait for its choice: concurrent tunings would time each
// other's launches and pick a shape at random.
struct BuildTuner {
    std::mutex mu;
    std::condition_variable cv;
    std::map<std::tuple<int, int, int, int>, int> best;
    std::set<std::tuple<int, int, int, int>> busy;
};
static BuildTuner& tuner() {
    static BuildTuner t;
    return t;
}

template <int DIM, typename R>
static void launch_build(Handle& H, int prev, const double* pu, const double* pp, R* mom, R* kdiag,
                         double* sdiag, double* f, bool outputs) {
    int dev = 0;
    GG_CUDA(cudaGetDevice(&dev));
    const double ppe = H.nel ? (double)H.np_in / (double)H.nel : 0.0;
    const int klass = ppe < 12 ? 0 : ppe < 24 ? 1 : ppe < 48 ? 2 : 3;
    const auto key = std::make_tuple(dev, DIM, (int)sizeof(R), klass);
    int shape = -1;
    bool tune = false;
    {
        std::unique_lock<std::mutex> lk(tuner().mu);
        for (;;) {
            auto it = tuner().best.find(key);
            if (it != tuner().best.end()) {
                shape = it->second;
                break;
            }
            if (!tuner().busy.count(key)) {
                tuner().busy.insert(key);
                tune = true;
                break;
            }
            tuner().cv.wait(lk);
        }
    }
    if (tune) {
        float best_ms = 1e30f;
        int best = 2;
        try {
            for (int rep = 0; rep < 2; rep++)
                for (int k = 0; k < kNumShapes; k++) {
                    GG_CUDA(cudaEventRecord(H.ev0, H.stream));
                    launch_build_shape<DIM, R>(k, H, prev, pu, pp, mom, kdiag, sdiag, f, outputs);
                    GG_CUDA(cudaEventRecord(H.ev1, H.stream));
                    GG_CUDA(cudaEventSynchronize(H.ev1));
                    float ms = 0.f;
                    GG_CUDA(cudaEventElapsedTime(&ms, H.ev0, H.ev1));
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = k;
                    }
                }
        } catch (...) {
            {
                std::lock_guard<std::mutex> lk(tuner().mu);
                tuner().busy.erase(key);
            }
            tuner().cv.notify_all();
            throw;
        }
        shape = best;
        {
            std::lock_guard<std::mutex> lk(tuner().mu);
            tuner().best[key] = shape;
            tuner().busy.erase(key);
        }
        tuner().cv.notify_all();
    }
    H.build_shape[sizeof(R) == 4 ? 1 : 0] = shape;
    launch_build_shape<DIM, R>(shape, H, prev, pu, pp, mom, kdiag, sdiag, f, outputs);
    gather_corners<DIM, R>(H, kdiag, f);
}

int build_operator(Handle& H, int precision, int prev, const double* d_prev_u,
                   const double* d_prev_p) {
    cudaStream_t st = H.stream;
    const int64_t nel = H.nel, nd = H.ndof;
    const int nm = H.nm;
    H.mom64.ensure(sizeof(double) * nm * nel);
    H.kdiag64.ensure(sizeof(double) * nd);
    H.sdiag.ensure(sizeof(double) * nel);
    H.f.ensure(sizeof(double) * nd);
    H.flag.ensure(sizeof(int32_t) * 4);
    // element corner terms of the diagonal and the force, summed per node after the build
    const int nen = 1 << H.dim;
    H.kcorner.ensure(sizeof(double) * nen * H.dim * nel);
    H.fcorner.ensure(sizeof(double) * 2 * nen * nel);
    upload_materials(H);
    GG_CUDA(cudaMemsetAsync(H.flag.p, 0, sizeof(int32_t) * 4, st));
    if (H.dim == 2)
        launch_build<2, double>(H, prev, d_prev_u, d_prev_p, H.mom64.as<double>(), H.kdiag64.as<double>(),
                                H.sdiag.as<double>(), H.f.as<double>(), true);
    else
        launch_build<3, double>(H, prev, d_prev_u, d_prev_p, H.mom64.as<double>(), H.kdiag64.as<double>(),
                                H.sdiag.as<double>(), H.f.as<double>(), true);
    if (precision == GG_PRECISION_MIXED) {
        H.mom32.ensure(sizeof(float) * nm * nel);
        H.kdiag32.ensure(sizeof(float) * nd);
        if (H.dim == 2)
            launch_build<2, float>(H, prev, d_prev_u, d_prev_p, H.mom32.as<float>(), H.kdiag32.as<float>(),
                                   nullptr, nullptr, false);
        else
            launch_build<3, float>(H, prev, d_prev_u, d_prev_p, H.mom32.as<float>(), H.kdiag32.as<float>(),
                                   nullptr, nullptr, false);
    }
    int32_t empty = 0;
    GG_CUDA(cudaMemcpyAsync(&empty, H.flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GG_CUDA(cudaStreamSynchronize(st));
    if (empty) return GG_ERR_EMPTY_CELL;
    return GG_OK;
}

}  // namespace gg
