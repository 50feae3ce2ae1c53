// gg_api2.cu -- C ABI: Picard, advection and the diagnostic / operator-access entry points.
#include <math.h>

#include <cstring>
#include <vector>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"
#include "gg_ops.cuh"

namespace gg {
int build_all(Handle& H, int precision, int prev, const double* d_u, const double* d_p);

namespace {
int grid(int64_t n) { return grid_for(n, 256); }

__global__ void k_add(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                      double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] + b[i];
}

__global__ void k_nodal_to_soa2(int64_t nnode, int dim, const double* __restrict__ in,
                                const uint8_t* __restrict__ bcmask, int zero_bc, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnode * dim;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = i / dim;
        const int c = (int)(i - n * dim);
        const bool fixed = zero_bc && ((bcmask[n] >> c) & 1);
        out[(int64_t)c * nnode + n] = fixed ? 0.0 : in[i];
    }
}

__global__ void k_soa_to_nodal2(int64_t nnode, int dim, const double* __restrict__ in, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnode * dim;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = i / dim;
        const int c = (int)(i - n * dim);
        out[i] = in[(int64_t)c * nnode + n];
    }
}

template <typename A, typename B>
__global__ void k_cvt(int64_t n, const A* __restrict__ a, B* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (B)a[i];
}

template <typename T>
__global__ void k_unsort(int64_t n, const int32_t* __restrict__ perm, const T* __restrict__ in, T* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[perm[i]] = in[i];
}

// ‖a − b‖², ‖a‖² partial sums (Picard residual), single block per 1024 entries + host sum
__global__ void k_diff_norms(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                             double* __restrict__ part) {
    __shared__ double s0[256], s1[256];
    double d2 = 0.0, a2 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double d = a[i] - b[i];
        d2 += d * d;
        a2 += a[i] * a[i];
    }
    s0[threadIdx.x] = d2;
    s1[threadIdx.x] = a2;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s0[threadIdx.x] += s0[threadIdx.x + o];
            s1[threadIdx.x] += s1[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s0[0];
        part[2 * blockIdx.x + 1] = s1[0];
    }
}

void nodal_in(Handle& H, const double* host, double* dst, bool zero_bc) {
    H.ftmp.ensure(sizeof(double) * H.ndof);
    GG_CUDA(cudaMemcpyAsync(H.ftmp.p, host, sizeof(double) * H.ndof, cudaMemcpyHostToDevice, H.stream));
    k_nodal_to_soa2<<<grid(H.ndof), 256, 0, H.stream>>>(H.nnode, H.dim, H.ftmp.as<double>(), H.bcmask.as<uint8_t>(),
                                                         zero_bc ? 1 : 0, dst);
    GG_CUDA(cudaGetLastError());
}

void nodal_out(Handle& H, const double* src, double* host) {
    H.ftmp.ensure(sizeof(double) * H.ndof);
    k_soa_to_nodal2<<<grid(H.ndof), 256, 0, H.stream>>>(H.nnode, H.dim, src, H.ftmp.as<double>());
    GG_CUDA(cudaGetLastError());
    GG_CUDA(cudaMemcpyAsync(host, H.ftmp.p, sizeof(double) * H.ndof, cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
}

int err(Handle& H, int code, const std::string& m) {
    H.err = m;
    return code;
}
}  // namespace

// prev_u = u + BC values (component-major), prev_p = q
void store_solution(Handle& H) {
    H.prev_u.ensure(sizeof(double) * H.ndof);
    H.prev_p.ensure(sizeof(double) * H.nel);
    k_add<<<grid(H.ndof), 256, 0, H.stream>>>(H.ndof, H.u.as<double>(), H.bcval.as<double>(), H.prev_u.as<double>());
    GG_CUDA(cudaGetLastError());
    GG_CUDA(cudaMemcpyAsync(H.prev_p.p, H.q.p, sizeof(double) * H.nel, cudaMemcpyDeviceToDevice, H.stream));
}

}  // namespace gg

using gg::Handle;
using namespace gg;

#define GG_TRY2(h, ...)                      \
    try {                                    \
        __VA_ARGS__                          \
    } catch (const gg::CudaError& ce) {      \
        (h)->H.err = ce.what;                \
        return GG_ERR_CUDA;                  \
    }

extern "C" {

int gg_picard(gg_handle* h, const gg_picard_params* pic, const gg_uzawa_params* prm, double* u, double* p,
              gg_picard_stats* stats) {
    if (!h || !pic || !prm || !u || !p || pic->max_iterations < 1) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.located) return gg::err(H, GG_ERR_STATE, "gg_locate has not succeeded");
    gg_picard_stats S{};
    int rc = GG_OK;
    GG_TRY2(h, {
        gg_uzawa_params up = *prm;
        gg_uzawa_stats us{};
        GG_CUDA(cudaMemsetAsync(H.q.p, 0, sizeof(double) * H.nel, H.stream));
        rc = gg::build_all(H, prm->precision, 0, nullptr, nullptr);
        if (rc == GG_OK) rc = gg::uzawa_solve(H, up, us);
        if (rc == GG_OK) {
            gg::store_solution(H);
            S.iterations = 1;
            S.outer_iterations += us.outer_iterations;
            S.inner_iterations += us.inner_iterations;
            S.solve_ms += us.solve_ms;
            H.picard_prev.ensure(sizeof(double) * H.ndof);
            const int nb = 256;
            H.picard_part.ensure(sizeof(double) * 2 * nb);
            std::vector<double> part(2 * nb);
            for (int it = 1; it < pic->max_iterations; it++) {
                GG_CUDA(cudaMemcpyAsync(H.picard_prev.p, H.u.p, sizeof(double) * H.ndof, cudaMemcpyDeviceToDevice,
                                        H.stream));
                rc = gg::build_all(H, prm->precision, 1, H.prev_u.as<double>(), H.prev_p.as<double>());
                if (rc != GG_OK) break;
                rc = gg::uzawa_solve(H, up, us);  // starts from the pressure in H.q
                if (rc != GG_OK) break;
                gg::store_solution(H);
                S.outer_iterations += us.outer_iterations;
                S.inner_iterations += us.inner_iterations;
                S.solve_ms += us.solve_ms;
                k_diff_norms<<<nb, 256, 0, H.stream>>>(H.ndof, H.u.as<double>(), H.picard_prev.as<double>(),
                                                       H.picard_part.as<double>());
                GG_CUDA(cudaMemcpyAsync(part.data(), H.picard_part.p, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost,
                                        H.stream));
                GG_CUDA(cudaStreamSynchronize(H.stream));
                double d2 = 0.0, a2 = 0.0;
                for (int b = 0; b < nb; b++) { d2 += part[2 * b]; a2 += part[2 * b + 1]; }
                S.residual = sqrt(d2) / sqrt(a2);
                S.iterations = it + 1;
                if (S.residual < pic->tolerance && it >= pic->min_iterations) { S.converged = 1; break; }
            }
        }
        if (H.have_solution || rc == GG_OK) {
            gg::nodal_out(H, H.prev_u.as<double>(), u);
            GG_CUDA(cudaMemcpyAsync(p, H.q.p, sizeof(double) * H.nel, cudaMemcpyDeviceToHost, H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
        }
        H.have_solution = rc == GG_OK;
    })
    if (stats) *stats = S;
    if (rc != GG_OK) gg::err(H, rc, "Picard iteration failed (status " + std::to_string(rc) + ")");
    return rc;
}

int gg_advect(gg_handle* h, double dt, int32_t order, const double* u, double* coords_out) {
    if (!h || (order != 1 && order != 2)) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (H.np == 0) return gg::err(H, GG_ERR_STATE, "points not set");
    int rc = GG_OK;
    GG_TRY2(h, {
        if (u) {
            H.prev_u.ensure(sizeof(double) * H.ndof);
            gg::nodal_in(H, u, H.prev_u.as<double>(), false);
        } else if (!H.have_solution) {
            return gg::err(H, GG_ERR_STATE, "no velocity to advect with");
        }
        rc = gg::advect(H, dt, order, H.prev_u.as<double>(), nullptr);
        if (coords_out) {
            GG_CUDA(cudaMemcpyAsync(coords_out, H.coords.p, sizeof(double) * H.np * H.dim, cudaMemcpyDeviceToHost,
                                    H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
        }
    })
    if (rc != GG_OK) gg::err(H, rc, "a material point left the mesh in the predictor stage");
    return rc;
}

int gg_courant_dt(gg_handle* h, const double* u, double* dt) {
    if (!h || !u || !dt) return GG_ERR_INVALID;
    Handle& H = h->H;
    double minsep = 1e300, vmax = 0.0;
    for (int d = 0; d < H.dim; d++) minsep = fmin(minsep, H.mk.sep[d]);
    for (int64_t n = 0; n < H.nnode; n++) {
        double v2 = 0.0;
        for (int c = 0; c < H.dim; c++) v2 += u[n * H.dim + c] * u[n * H.dim + c];
        vmax = fmax(vmax, v2);
    }
    *dt = vmax == 0.0 ? 0.0 : 0.5 * minsep / sqrt(vmax);
    return GG_OK;
}

int gg_get_point_viscosity(gg_handle* h, double* eta) {
    if (!h || !eta) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built) return gg::err(H, GG_ERR_STATE, "operator not built");
    GG_TRY2(h, {
        H.ftmp.ensure(sizeof(double) * (H.np > H.ndof ? H.np : H.ndof));
        gg::k_unsort<double><<<grid(H.np_in), 256, 0, H.stream>>>(H.np_in, H.perm.as<int32_t>(), H.eta_s.as<double>(),
                                                                  H.ftmp.as<double>());
        GG_CUDA(cudaMemcpyAsync(eta, H.ftmp.p, sizeof(double) * H.np, cudaMemcpyDeviceToHost, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
    })
    return GG_OK;
}

int gg_get_point_yield(gg_handle* h, double* increment, uint8_t* yielded) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built) return gg::err(H, GG_ERR_STATE, "operator not built");
    GG_TRY2(h, {
        H.ftmp.ensure(sizeof(double) * (H.np > H.ndof ? H.np : H.ndof));
        if (increment) {
            gg::k_unsort<double><<<grid(H.np_in), 256, 0, H.stream>>>(H.np_in, H.perm.as<int32_t>(),
                                                                      H.incr_s.as<double>(), H.ftmp.as<double>());
            GG_CUDA(cudaMemcpyAsync(increment, H.ftmp.p, sizeof(double) * H.np, cudaMemcpyDeviceToHost, H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
        }
        if (yielded) {
            gg::k_unsort<uint8_t><<<grid(H.np_in), 256, 0, H.stream>>>(H.np_in, H.perm.as<int32_t>(),
                                                                       H.yld_s.as<uint8_t>(), H.ftmp.as<uint8_t>());
            GG_CUDA(cudaMemcpyAsync(yielded, H.ftmp.p, H.np, cudaMemcpyDeviceToHost, H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
        }
    })
    return GG_OK;
}

int gg_get_moments(gg_handle* h, double* moments, int32_t* n_moments) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (n_moments) *n_moments = H.nm;
    if (!moments) return GG_OK;
    if (!H.built) return gg::err(H, GG_ERR_STATE, "operator not built");
    GG_TRY2(h, {
        GG_CUDA(cudaMemcpyAsync(moments, H.mom64.p, sizeof(double) * H.nm * H.nel, cudaMemcpyDeviceToHost, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
    })
    return GG_OK;
}

int gg_apply_K(gg_handle* h, int32_t precision, const double* x, double* y) {
    if (!h || !x || !y) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built) return gg::err(H, GG_ERR_STATE, "operator not built");
    if (precision == GG_PRECISION_MIXED && H.built_precision != GG_PRECISION_MIXED)
        return gg::err(H, GG_ERR_STATE, "operator built without the FP32 moments");
    GG_TRY2(h, {
        H.vstar.ensure(sizeof(double) * H.ndof);
        H.ub.ensure(sizeof(double) * H.ndof);
        gg::nodal_in(H, x, H.vstar.as<double>(), true);
        GG_CUDA(cudaMemsetAsync(H.ub.p, 0, sizeof(double) * H.ndof, H.stream));
        if (precision == GG_PRECISION_FP64) {
            gg::apply_K<double>(H.mk, H.mom64.as<double>(), H.bcmask.as<uint8_t>(), H.vstar.as<double>(),
                                H.ub.as<double>(), H.stream);
        } else {
            H.r32.ensure(sizeof(float) * H.ndof);
            H.Ap32.ensure(sizeof(float) * H.ndof);
            gg::k_cvt<double, float><<<grid(H.ndof), 256, 0, H.stream>>>(H.ndof, H.vstar.as<double>(), H.r32.as<float>());
            GG_CUDA(cudaMemsetAsync(H.Ap32.p, 0, sizeof(float) * H.ndof, H.stream));
            gg::apply_K<float>(H.mk, H.mom32.as<float>(), H.bcmask.as<uint8_t>(), H.r32.as<float>(), H.Ap32.as<float>(),
                               H.stream);
            gg::k_cvt<float, double><<<grid(H.ndof), 256, 0, H.stream>>>(H.ndof, H.Ap32.as<float>(), H.ub.as<double>());
        }
        gg::nodal_out(H, H.ub.as<double>(), y);
    })
    return GG_OK;
}

int gg_learned_train(gg_handle* h, const gg_learn_params* params, gg_learn_stats* stats) {
    if (!h || !params) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built || H.built_precision != GG_PRECISION_MIXED)
        return gg::err(H, GG_ERR_STATE, "training needs an operator built with GG_PRECISION_MIXED");
    gg_learn_stats S{};
    int rc = GG_OK;
    GG_TRY2(h, {
        for (gg::DBuf* b : {&H.r32, &H.cgr32, &H.z32, &H.p32, &H.Ap32, &H.e32, &H.mg_xs, &H.mg_xk, &H.mg_xt})
            b->ensure(sizeof(float) * H.ndof);
        H.qtmp.ensure(sizeof(double) * H.nel);
        H.ftmp.ensure(sizeof(double) * H.ndof);
        gg::prepare_krylov_scratch(H);
        rc = gg::learned_train(H, *params, S);
    })
    if (stats) *stats = S;
    if (rc != GG_OK) gg::err(H, rc, "learned training failed (status " + std::to_string(rc) + ")");
    return rc;
}

int gg_learned_weights(gg_handle* h, float* weights, int32_t* n) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (n) *n = (int32_t)gg::learned_param_count(H);
    if (!weights) return GG_OK;
    if (!H.nn_ready) return gg::err(H, GG_ERR_STATE, "no trained network");
    GG_TRY2(h, { gg::learned_get_weights(H, weights); })
    return GG_OK;
}

int gg_learned_set_weights(gg_handle* h, int32_t level, const float* weights, int32_t n) {
    if (!h || !weights) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (n != (int32_t)gg::learned_param_count(H)) return gg::err(H, GG_ERR_INVALID, "parameter count");
    if (!H.built || H.built_precision != GG_PRECISION_MIXED)
        return gg::err(H, GG_ERR_STATE, "needs an operator built with GG_PRECISION_MIXED");
    int rc = GG_OK;
    GG_TRY2(h, {
        rc = gg::learned_set_level(H, level);
        if (rc == GG_OK) gg::learned_set_weights(H, weights);
    })
    return rc;
}

int gg_learned_eval(gg_handle* h, int32_t level, int32_t batch, const float* inputs, const float* targets,
                    const float* weights, float* outputs, float* gradient, double* loss, int32_t* grid_nodes) {
    if (!h || batch < 1 || !inputs || !targets || !weights || !outputs || !gradient || !loss || !grid_nodes)
        return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built || H.built_precision != GG_PRECISION_MIXED)
        return gg::err(H, GG_ERR_STATE, "needs an operator built with GG_PRECISION_MIXED");
    int rc = GG_OK;
    GG_TRY2(h, {
        rc = gg::learned_set_level(H, level);
        if (rc == GG_OK) {
            const int32_t nodes = (int32_t)H.mg[H.nn_level]->nnode;
            if (*grid_nodes != nodes) {
                rc = gg::err(H, GG_ERR_INVALID, "buffers hold " + std::to_string(*grid_nodes) + " nodes, level " +
                                                    std::to_string(H.nn_level) + " has " + std::to_string(nodes));
            } else {
                rc = gg::learned_eval(H, batch, inputs, targets, weights, outputs, gradient, loss);
            }
            *grid_nodes = nodes;
        }
    })
    return rc;
}

int gg_set_weights(gg_handle* h, const gg_weights* w) {
    if (!h || !w) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (w->mode != GG_WEIGHTS_CONSTANT && w->mode != GG_WEIGHTS_DVC)
        return gg::err(H, GG_ERR_INVALID, "weights mode");
    if (w->mode == GG_WEIGHTS_DVC) {
        const int nz = H.dim == 3 ? w->resolution[2] : 1;
        if (w->resolution[0] < 1 || w->resolution[1] < 1 || nz < 1 || w->resolution[0] > 64 || w->resolution[1] > 64 ||
            nz > 64 || w->resolution[0] * w->resolution[1] * nz > 1024)
            return gg::err(H, GG_ERR_INVALID, "DVC resolution: at most 64 per axis and 1024 cells per element");
    }
    H.weights = *w;
    // the integration points change: locate again before the next build
    H.located = false;
    H.built = false;
    H.dvc_valid = false;
    return GG_OK;
}

int gg_population_control(gg_handle* h, const gg_pcdvc_params* prm, gg_pcdvc_stats* stats) {
    if (!h || !prm) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (H.weights.mode != GG_WEIGHTS_DVC) return gg::err(H, GG_ERR_STATE, "population control needs GG_WEIGHTS_DVC");
    if (!H.located) return gg::err(H, GG_ERR_STATE, "gg_locate has not succeeded");
    int rc = GG_OK;
    gg_pcdvc_stats st{};
    GG_TRY2(h, {
        GG_CUDA(cudaEventRecord(H.ev0, H.stream));
        rc = gg::dvc_update(H, prm, &st);
        GG_CUDA(cudaEventRecord(H.ev1, H.stream));
        GG_CUDA(cudaEventSynchronize(H.ev1));
        float ms = 0.f;
        GG_CUDA(cudaEventElapsedTime(&ms, H.ev0, H.ev1));
        st.ms = ms;
    })
    H.built = false;
    if (rc != GG_OK) H.located = false;
    if (stats) *stats = st;
    return rc;
}

int gg_point_count(gg_handle* h, int64_t* n) {
    if (!h || !n) return GG_ERR_INVALID;
    *n = h->H.np;
    return GG_OK;
}

int gg_get_points(gg_handle* h, double* coords, int32_t* material, double* plastic_strain) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (H.np == 0) return gg::err(H, GG_ERR_STATE, "points not set");
    GG_TRY2(h, {
        if (coords)
            GG_CUDA(cudaMemcpyAsync(coords, H.coords.p, sizeof(double) * H.np * H.dim, cudaMemcpyDeviceToHost, H.stream));
        if (material)
            GG_CUDA(cudaMemcpyAsync(material, H.mat_in.p, sizeof(int32_t) * H.np, cudaMemcpyDeviceToHost, H.stream));
        if (plastic_strain)
            GG_CUDA(cudaMemcpyAsync(plastic_strain, H.ps_in.p, sizeof(double) * H.np, cudaMemcpyDeviceToHost, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
    })
    return GG_OK;
}

}  // extern "C"

namespace gg {
namespace {
// sorted integration points → point order; constant weights from the element counts
__global__ void k_int_points(int64_t np, int dim, const int32_t* __restrict__ perm, const int32_t* __restrict__ cell_s,
                             const int32_t* __restrict__ offsets, const double* __restrict__ xi_s,
                             const double* __restrict__ w_s, double* __restrict__ xi, double* __restrict__ w) {
    const double wscale = (double)(1 << dim);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = perm[i];
        for (int d = 0; d < dim; d++) xi[(int64_t)p * dim + d] = xi_s[(int64_t)d * np + i];
        const int32_t e = cell_s[i];
        w[p] = w_s ? w_s[i] : wscale / (double)(offsets[e + 1] - offsets[e]);
    }
}
}  // namespace
}  // namespace gg

extern "C" {

int gg_get_integration_points(gg_handle* h, double* xi, double* weight) {
    if (!h || !xi || !weight) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.located) return gg::err(H, GG_ERR_STATE, "gg_locate has not succeeded");
    GG_TRY2(h, {
        DBuf dx, dw;
        dx.ensure(sizeof(double) * H.np * H.dim);
        dw.ensure(sizeof(double) * H.np);
        gg::k_int_points<<<gg::grid_for(H.np, 256), 256, 0, H.stream>>>(
            H.np, H.dim, H.perm.as<int32_t>(), H.cell_s.as<int32_t>(), H.offsets.as<int32_t>(), H.xi_s.as<double>(),
            H.weights.mode == GG_WEIGHTS_DVC && H.dvc_valid ? H.w_s.as<double>() : nullptr, dx.as<double>(),
            dw.as<double>());
        GG_CUDA(cudaGetLastError());
        GG_CUDA(cudaMemcpyAsync(xi, dx.p, sizeof(double) * H.np * H.dim, cudaMemcpyDeviceToHost, H.stream));
        GG_CUDA(cudaMemcpyAsync(weight, dw.p, sizeof(double) * H.np, cudaMemcpyDeviceToHost, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
    })
    return GG_OK;
}

int gg_check_grid_barrier_timeout(int32_t spin_limit, int32_t* blocks_gave_up) {
    if (!blocks_gave_up) return GG_ERR_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GG_ERR_NO_DEVICE;
    try {
        int g = 0;
        const int rc = gg::check_barrier_timeout(spin_limit, &g);
        *blocks_gave_up = g;
        return rc;
    } catch (const gg::CudaError&) {
        return GG_ERR_CUDA;
    }
}

int gg_time_grid_barrier(int32_t blocks_per_sm, int32_t iters, double* us_per_barrier) {
    if (!us_per_barrier) return GG_ERR_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GG_ERR_NO_DEVICE;
    try {
        return gg::time_grid_barrier(blocks_per_sm, iters, us_per_barrier);
    } catch (const gg::CudaError&) {
        return GG_ERR_CUDA;
    }
}

int gg_time_apply(gg_handle* h, int32_t precision, int32_t reps, double* ms_per_launch) {
    if (!h || !ms_per_launch || reps < 1) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built) return gg::err(H, GG_ERR_STATE, "operator not built");
    if (precision == GG_PRECISION_MIXED && H.built_precision != GG_PRECISION_MIXED)
        return gg::err(H, GG_ERR_STATE, "operator built without the FP32 moments");
    GG_TRY2(h, {
        H.vstar.ensure(sizeof(double) * H.ndof);
        H.ub.ensure(sizeof(double) * H.ndof);
        // input: the force vector (zero on BC rows), output accumulates
        GG_CUDA(cudaMemcpyAsync(H.vstar.p, H.f.p, sizeof(double) * H.ndof, cudaMemcpyDeviceToDevice, H.stream));
        GG_CUDA(cudaMemsetAsync(H.ub.p, 0, sizeof(double) * H.ndof, H.stream));
        if (precision == GG_PRECISION_MIXED) {
            H.r32.ensure(sizeof(float) * H.ndof);
            H.Ap32.ensure(sizeof(float) * H.ndof);
            gg::k_cvt<double, float><<<grid(H.ndof), 256, 0, H.stream>>>(H.ndof, H.vstar.as<double>(), H.r32.as<float>());
            GG_CUDA(cudaMemsetAsync(H.Ap32.p, 0, sizeof(float) * H.ndof, H.stream));
        }
        auto launch = [&]() {
            if (precision == GG_PRECISION_MIXED)
                gg::apply_K<float>(H.mk, H.mom32.as<float>(), H.bcmask.as<uint8_t>(), H.r32.as<float>(),
                                   H.Ap32.as<float>(), H.stream);
            else
                gg::apply_K<double>(H.mk, H.mom64.as<double>(), H.bcmask.as<uint8_t>(), H.vstar.as<double>(),
                                    H.ub.as<double>(), H.stream);
        };
        launch();  // warm-up
        GG_CUDA(cudaEventRecord(H.ev0, H.stream));
        for (int i = 0; i < reps; i++) launch();
        GG_CUDA(cudaEventRecord(H.ev1, H.stream));
        GG_CUDA(cudaEventSynchronize(H.ev1));
        float ms = 0.f;
        GG_CUDA(cudaEventElapsedTime(&ms, H.ev0, H.ev1));
        *ms_per_launch = (double)ms / reps;
    })
    return GG_OK;
}

int gg_get_coarse_inverse(gg_handle* h, int64_t* n, float* inverse, double* op) {
    if (!h || !n) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built) return gg::err(H, GG_ERR_STATE, "operator not built");
    int rc = GG_OK;
    GG_TRY2(h, { rc = gg::coarse_inverse_copy(H, n, inverse, op); })
    return rc;
}

int gg_apply_G(gg_handle* h, const double* p, double* y) {
    if (!h || !p || !y) return GG_ERR_INVALID;
    Handle& H = h->H;
    GG_TRY2(h, {
        H.qtmp.ensure(sizeof(double) * H.nel);
        H.ub.ensure(sizeof(double) * H.ndof);
        GG_CUDA(cudaMemcpyAsync(H.qtmp.p, p, sizeof(double) * H.nel, cudaMemcpyHostToDevice, H.stream));
        gg::apply_G(H, H.qtmp.as<double>(), H.ub.as<double>(), H.stream);
        gg::nodal_out(H, H.ub.as<double>(), y);
    })
    return GG_OK;
}

int gg_apply_GT(gg_handle* h, const double* u, double* q) {
    if (!h || !u || !q) return GG_ERR_INVALID;
    Handle& H = h->H;
    GG_TRY2(h, {
        H.qtmp.ensure(sizeof(double) * H.nel);
        H.vstar.ensure(sizeof(double) * H.ndof);
        gg::nodal_in(H, u, H.vstar.as<double>(), true);
        gg::apply_GT(H, H.vstar.as<double>(), H.qtmp.as<double>(), H.stream);
        GG_CUDA(cudaMemcpyAsync(q, H.qtmp.p, sizeof(double) * H.nel, cudaMemcpyDeviceToHost, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
    })
    return GG_OK;
}

int gg_get_rhs(gg_handle* h, double* f, double* hvec) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built) return gg::err(H, GG_ERR_STATE, "operator not built");
    GG_TRY2(h, {
        if (f) gg::nodal_out(H, H.f.as<double>(), f);
        if (hvec) {
            GG_CUDA(cudaMemcpyAsync(hvec, H.hvec.p, sizeof(double) * H.nel, cudaMemcpyDeviceToHost, H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
        }
    })
    return GG_OK;
}

int gg_get_diagonals(gg_handle* h, double* k_diag, double* schur_diag) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built) return gg::err(H, GG_ERR_STATE, "operator not built");
    GG_TRY2(h, {
        if (k_diag) gg::nodal_out(H, H.kdiag64.as<double>(), k_diag);
        if (schur_diag) {
            GG_CUDA(cudaMemcpyAsync(schur_diag, H.sdiag.p, sizeof(double) * H.nel, cudaMemcpyDeviceToHost, H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
        }
    })
    return GG_OK;
}

}  // extern "C"
