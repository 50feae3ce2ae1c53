// gg_api.cu -- the C ABI (include/gale_gpu.h) over the sm_100a kernels.
//
// Every entry point validates its arguments, runs on the handle's stream and converts
// CUDA failures into GG_ERR_CUDA with a message; nothing aborts the host process.
// Host arrays are node-major (FeVariable dof layout); device arrays are component-major.
#include <math.h>
#include <stdio.h>

#include <cstring>
#include <new>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"
#include "gg_ops.cuh"

namespace gg {

int num_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    }
    return n;
}

namespace {

__global__ void k_nodal_to_soa(int64_t nnode, int dim, const double* __restrict__ in,
                               const uint8_t* __restrict__ bcmask, int zero_bc, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnode * dim;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = i / dim;
        const int c = (int)(i - n * dim);
        const bool fixed = zero_bc && ((bcmask[n] >> c) & 1);
        out[(int64_t)c * nnode + n] = fixed ? 0.0 : in[i];
    }
}

__global__ void k_soa_to_nodal(int64_t nnode, int dim, const double* __restrict__ in,
                               const double* __restrict__ add, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnode * dim;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = i / dim;
        const int c = (int)(i - n * dim);
        const int64_t j = (int64_t)c * nnode + n;
        out[i] = in[j] + (add ? add[j] : 0.0);
    }
}

// f ← f − K_fb u_b on free rows, 0 on BC rows (StiffnessMatrix.cxx:2091-2117)
__global__ void k_finish_rhs(int64_t n, int64_t nnode, const uint8_t* __restrict__ bcmask,
                             const double* __restrict__ kub, double* __restrict__ f) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i / nnode);
        const bool fixed = (bcmask[i - (int64_t)c * nnode] >> c) & 1;
        f[i] = fixed ? 0.0 : f[i] - kub[i];
    }
}

__global__ void k_neg(int64_t n, double* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] = -x[i];
}

template <typename A, typename B>
__global__ void k_convert(int64_t n, const A* __restrict__ a, B* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (B)a[i];
}

template <typename T>
__global__ void k_unsort(int64_t n, const int32_t* __restrict__ perm, const T* __restrict__ in,
                         T* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[perm[i]] = in[i];
}

// Element gradient on the 2^dim Gauss swarm, as _GradientStiffnessMatrixTerm_AssembleElement
// integrates it (GradientStiffnessMatrixTerm.cxx:213-246), for an element of size h.
void gauss_G(int dim, const double* h, double Ge[8][3]) {
    const double g = 1.0 / sqrt(3.0);
    for (int a = 0; a < 8; a++)
        for (int d = 0; d < 3; d++) Ge[a][d] = 0.0;
    double detJ = 1.0;
    for (int d = 0; d < dim; d++) detJ *= 0.5 * h[d];
    for (int q = 0; q < (1 << dim); q++) {
        double xi[3] = {(q & 1) ? g : -g, (q & 2) ? g : -g, (q & 4) ? g : -g};
        for (int a = 0; a < (1 << dim); a++)
            for (int d = 0; d < dim; d++) {
                double v = (dim == 2 ? 0.25 : 0.125) * (((a >> d) & 1) ? 1.0 : -1.0);
                for (int o = 0; o < dim; o++)
                    if (o != d) v *= 1.0 + (((a >> o) & 1) ? xi[o] : -xi[o]);
                const double gnx = v / (0.5 * h[d]);
                Ge[a][d] += 1.0 * (-detJ) * (gnx * 1.0);
            }
    }
}

}  // namespace

int set_error(Handle& H, int code, const std::string& msg) {
    H.err = msg;
    return code;
}

MeshK make_mesh(const gg_mesh_desc& d) {
    MeshK mk{};
    mk.dim = d.dim;
    mk.nel = 1;
    mk.nnode = 1;
    for (int i = 0; i < 3; i++) {
        const bool used = i < d.dim;
        mk.n[i] = used ? d.elements[i] : 1;
        mk.nn[i] = used ? d.elements[i] + 1 : 1;
        mk.min[i] = used ? d.min[i] : 0.0;
        mk.max[i] = used ? d.max[i] : 0.0;
        mk.sep[i] = used ? (d.max[i] - d.min[i]) / d.elements[i] : 1.0;
        mk.h[i] = used ? (d.max[i] - d.min[i]) / d.elements[i] : 2.0;
    }
    for (int i = 0; i < d.dim; i++) {
        mk.nel *= mk.n[i];
        mk.nnode *= mk.nn[i];
    }
    mk.detJ = 1.0;
    for (int i = 0; i < d.dim; i++) mk.detJ *= 0.5 * mk.h[i];
    for (int i = 0; i < 3; i++) mk.kappa[i] = i < d.dim ? 2.0 / (mk.h[i] * (double)(1 << d.dim)) : 0.0;
    gauss_G(d.dim, mk.h, mk.Ge);
    return mk;
}

}  // namespace gg

using gg::Handle;

#define GG_TRY(h, ...)                                                       \
    try {                                                                    \
        __VA_ARGS__                                                          \
    } catch (const gg::CudaError& ce) {                                      \
        (h)->H.err = ce.what;                                                \
        return GG_ERR_CUDA;                                                  \
    } catch (const std::bad_alloc&) {                                        \
        (h)->H.err = "host allocation failed";                               \
        return GG_ERR_CUDA;                                                  \
    }

static int grid(int64_t n) { return gg::grid_for(n, 256); }

extern "C" {

const char* gg_version(void) { return "gale_b200 0.1 (sm_100a)"; }

const char* gg_last_error(const gg_handle* h) { return h ? h->H.err.c_str() : "null handle"; }

int gg_create(const gg_mesh_desc* mesh, gg_handle** out) {
    if (!mesh || !out) return GG_ERR_INVALID;
    *out = nullptr;
    if (mesh->dim != 2 && mesh->dim != 3) return GG_ERR_INVALID;
    for (int d = 0; d < mesh->dim; d++) {
        if (mesh->elements[d] < 1 || !(mesh->max[d] > mesh->min[d])) return GG_ERR_INVALID;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return GG_ERR_NO_DEVICE;
    gg_handle* h = new (std::nothrow) gg_handle();
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    try {
        H.desc = *mesh;
        H.mk = gg::make_mesh(*mesh);
        H.dim = mesh->dim;
        H.nm = mesh->dim == 2 ? gg::n_moments<2>() : gg::n_moments<3>();
        H.nel = H.mk.nel;
        H.nnode = H.mk.nnode;
        H.ndof = H.nnode * H.dim;
        if (H.nel >= (int64_t)INT32_MAX) throw gg::CudaError(cudaErrorInvalidValue, "mesh too large", __FILE__, __LINE__);
        GG_CUDA(cudaStreamCreateWithFlags(&H.stream, cudaStreamNonBlocking));
        GG_CUDA(cudaEventCreate(&H.ev0));
        GG_CUDA(cudaEventCreate(&H.ev1));
        GG_CUDA(cudaEventCreate(&H.evf0));
        GG_CUDA(cudaEventCreate(&H.evf1));
        H.bcmask.ensure(H.nnode);
        H.bcval.ensure(sizeof(double) * H.ndof);
        GG_CUDA(cudaMemsetAsync(H.bcmask.p, 0, H.nnode, H.stream));
        GG_CUDA(cudaMemsetAsync(H.bcval.p, 0, sizeof(double) * H.ndof, H.stream));
        H.nfree = H.ndof;
        H.force.g_hat[1] = -1.0;
        H.hvec.ensure(sizeof(double) * H.nel);
        H.q.ensure(sizeof(double) * H.nel);
        GG_CUDA(cudaMemsetAsync(H.q.p, 0, sizeof(double) * H.nel, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
    } catch (const gg::CudaError& ce) {
        delete h;
        return GG_ERR_CUDA;
    }
    *out = h;
    return GG_OK;
}

int gg_destroy(gg_handle* h) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (H.stream) cudaStreamSynchronize(H.stream);
    gg::release_graphs(H);
    if (H.h_scal) cudaFreeHost(H.h_scal);
    if (H.ev0) cudaEventDestroy(H.ev0);
    if (H.ev1) cudaEventDestroy(H.ev1);
    if (H.evf0) cudaEventDestroy(H.evf0);
    if (H.evf1) cudaEventDestroy(H.evf1);
    if (H.stream) cudaStreamDestroy(H.stream);
    delete h;
    return GG_OK;
}

int gg_set_velocity_bc(gg_handle* h, const gg_velocity_bc* bc) {
    if (!h || !bc) return GG_ERR_INVALID;
    Handle& H = h->H;
    GG_TRY(h, {
        const int dim = H.dim;
        std::vector<uint8_t> mask(H.nnode, 0);
        std::vector<double> val(H.ndof, 0.0);
        int64_t nfixed = 0;
        for (int64_t n = 0; n < H.nnode; n++) {
            const int idx[3] = {(int)(n % H.mk.nn[0]), (int)((n / H.mk.nn[0]) % H.mk.nn[1]),
                                (int)(n / ((int64_t)H.mk.nn[0] * H.mk.nn[1]))};
            for (int wall = 0; wall < 2 * dim; wall++) {
                const int ax = wall / 2;
                const bool on = (wall & 1) ? idx[ax] == H.mk.n[ax] : idx[ax] == 0;
                if (!on) continue;
                for (int c = 0; c < dim; c++)
                    if (bc->fixed[wall][c]) {
                        mask[n] |= (uint8_t)(1u << c);
                        val[(int64_t)c * H.nnode + n] = bc->value[wall][c];
                    }
            }
            for (int c = 0; c < dim; c++) nfixed += (mask[n] >> c) & 1;
        }
        H.nfree = H.ndof - nfixed;
        GG_CUDA(cudaMemcpyAsync(H.bcmask.p, mask.data(), H.nnode, cudaMemcpyHostToDevice, H.stream));
        GG_CUDA(cudaMemcpyAsync(H.bcval.p, val.data(), sizeof(double) * H.ndof, cudaMemcpyHostToDevice, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
        H.has_bc = true;
        H.built = false;
        gg::release_graphs(H);
    })
    return GG_OK;
}

int gg_set_velocity_bc_nodes(gg_handle* h, const uint8_t* fixed, const double* values) {
    if (!h || !fixed || !values) return GG_ERR_INVALID;
    Handle& H = h->H;
    GG_TRY(h, {
        const int dim = H.dim;
        std::vector<uint8_t> mask(H.nnode, 0);
        std::vector<double> val(H.ndof, 0.0);
        int64_t nfixed = 0;
        for (int64_t n = 0; n < H.nnode; n++) {
            mask[n] = (uint8_t)(fixed[n] & ((1u << dim) - 1u));
            for (int c = 0; c < dim; c++)
                if ((mask[n] >> c) & 1) {
                    val[(int64_t)c * H.nnode + n] = values[n * dim + c];
                    nfixed++;
                }
        }
        H.nfree = H.ndof - nfixed;
        GG_CUDA(cudaMemcpyAsync(H.bcmask.p, mask.data(), H.nnode, cudaMemcpyHostToDevice, H.stream));
        GG_CUDA(cudaMemcpyAsync(H.bcval.p, val.data(), sizeof(double) * H.ndof, cudaMemcpyHostToDevice, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
        H.has_bc = true;
        H.built = false;
        gg::release_graphs(H);
    })
    return GG_OK;
}

int gg_set_materials(gg_handle* h, int32_t n, const gg_material* mats) {
    if (!h || !mats || n < 1 || n > GG_MAX_MATERIALS) return h ? gg::set_error(h->H, GG_ERR_INVALID, "material count") : GG_ERR_INVALID;
    for (int i = 0; i < n; i++) {
        if (mats[i].n_rheologies < 0 || mats[i].n_rheologies > GG_MAX_RHEOLOGIES)
            return gg::set_error(h->H, GG_ERR_INVALID, "rheology count");
        // DruckerPrager's HydrostaticTerm (DruckerPrager.cxx:327-332) adds a lithostatic
        // pressure this library does not evaluate: refused rather than silently dropped
        for (int k = 0; k < mats[i].n_rheologies; k++)
            if (mats[i].rheology[k].hydrostatic_term)
                return gg::set_error(h->H, GG_ERR_INVALID, "DruckerPrager HydrostaticTerm is not supported");
    }
    h->H.materials.assign(mats, mats + n);
    h->H.n_materials = n;
    h->H.built = false;
    return GG_OK;
}

int gg_set_points(gg_handle* h, int64_t n, const double* coords, const int32_t* material,
                  const double* plastic_strain) {
    if (!h || !coords || n < 1 || n >= (int64_t)INT32_MAX) return h ? gg::set_error(h->H, GG_ERR_INVALID, "point count") : GG_ERR_INVALID;
    Handle& H = h->H;
    int32_t maxm = 0;
    if (material) {
        for (int64_t i = 0; i < n; i++) {
            if (material[i] < 0 || material[i] >= GG_MAX_MATERIALS)
                return gg::set_error(H, GG_ERR_INVALID, "material index out of range");
            if (material[i] > maxm) maxm = material[i];
        }
    }
    H.max_material = maxm;
    GG_TRY(h, {
        const int dim = H.dim;
        H.np = n;
        H.coords.ensure(sizeof(double) * n * dim);
        H.mat_in.ensure(sizeof(int32_t) * n);
        H.ps_in.ensure(sizeof(double) * n);
        for (gg::DBuf* b : {&H.cell, &H.perm, &H.cell_s, &H.mat_s}) b->ensure(sizeof(int32_t) * n);
        for (gg::DBuf* b : {&H.ps_s, &H.eta_s, &H.incr_s}) b->ensure(sizeof(double) * n);
        H.xi_s.ensure(sizeof(double) * n * dim);
        H.yld_s.ensure(n);
        GG_CUDA(cudaMemcpyAsync(H.coords.p, coords, sizeof(double) * n * dim, cudaMemcpyHostToDevice, H.stream));
        if (material)
            GG_CUDA(cudaMemcpyAsync(H.mat_in.p, material, sizeof(int32_t) * n, cudaMemcpyHostToDevice, H.stream));
        else
            GG_CUDA(cudaMemsetAsync(H.mat_in.p, 0, sizeof(int32_t) * n, H.stream));
        if (plastic_strain)
            GG_CUDA(cudaMemcpyAsync(H.ps_in.p, plastic_strain, sizeof(double) * n, cudaMemcpyHostToDevice, H.stream));
        else
            GG_CUDA(cudaMemsetAsync(H.ps_in.p, 0, sizeof(double) * n, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
        H.located = false;
        H.built = false;
        H.dvc_valid = false;
    })
    return GG_OK;
}

int gg_set_temperature(gg_handle* h, const double* T) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    GG_TRY(h, {
        if (T) {
            H.T.ensure(sizeof(double) * H.nnode);
            GG_CUDA(cudaMemcpyAsync(H.T.p, T, sizeof(double) * H.nnode, cudaMemcpyHostToDevice, H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
            H.has_T = true;
        } else {
            H.has_T = false;
        }
        H.built = false;
    })
    return GG_OK;
}

int gg_set_body_force(gg_handle* h, const gg_body_force* f) {
    if (!h || !f) return GG_ERR_INVALID;
    Handle& H = h->H;
    H.force = *f;
    double nrm = 0.0;
    for (int d = 0; d < H.dim; d++) nrm += f->g_hat[d] * f->g_hat[d];
    nrm = sqrt(nrm);
    for (int d = 0; d < 3; d++) H.force.g_hat[d] = (d < H.dim && nrm > 0) ? f->g_hat[d] / nrm : 0.0;
    H.built = false;
    return GG_OK;
}

int gg_locate(gg_handle* h, uint32_t* owning_cell) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (H.np == 0) return gg::set_error(H, GG_ERR_STATE, "points not set");
    int64_t outside = 0;
    int rc = GG_OK;
    GG_TRY(h, {
        outside = gg::locate_and_sort(H);
        H.np_in = H.np - outside;
        H.dvc_valid = false;
        if (!outside && H.weights.mode == GG_WEIGHTS_DVC) rc = gg::dvc_update(H, nullptr, nullptr);
        if (owning_cell) {
            GG_CUDA(cudaMemcpyAsync(owning_cell, H.cell.p, sizeof(uint32_t) * H.np, cudaMemcpyDeviceToHost, H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
        }
    })
    H.located = outside == 0 && rc == GG_OK;
    H.built = false;
    if (outside) return gg::set_error(H, GG_ERR_OUT_OF_DOMAIN, std::to_string(outside) + " material points outside the mesh");
    return rc;
}

}  // extern "C"

namespace gg {
// Upload a nodal host vector (node-major) into a component-major device buffer.
static void upload_nodal(Handle& H, const double* host, DBuf& dst, bool zero_bc) {
    H.ftmp.ensure(sizeof(double) * H.ndof);
    dst.ensure(sizeof(double) * H.ndof);
    GG_CUDA(cudaMemcpyAsync(H.ftmp.p, host, sizeof(double) * H.ndof, cudaMemcpyHostToDevice, H.stream));
    k_nodal_to_soa<<<grid(H.ndof), 256, 0, H.stream>>>(H.nnode, H.dim, H.ftmp.as<double>(), H.bcmask.as<uint8_t>(),
                                                        zero_bc ? 1 : 0, dst.as<double>());
    GG_CUDA(cudaGetLastError());
}
static void download_nodal(Handle& H, const double* dsrc, const double* add, double* host) {
    H.ftmp.ensure(sizeof(double) * H.ndof);
    k_soa_to_nodal<<<grid(H.ndof), 256, 0, H.stream>>>(H.nnode, H.dim, dsrc, add, H.ftmp.as<double>());
    GG_CUDA(cudaGetLastError());
    GG_CUDA(cudaMemcpyAsync(host, H.ftmp.p, sizeof(double) * H.ndof, cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
}

void download_solution(Handle& H, double* u, double* p) {
    store_solution(H);
    download_nodal(H, H.u.as<double>(), H.bcval.as<double>(), u);
    GG_CUDA(cudaMemcpyAsync(p, H.q.p, sizeof(double) * H.nel, cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
    H.have_solution = true;
}

// Operator build + Dirichlet elimination; device previous solution pointers (nullable).
int build_all(Handle& H, int precision, int prev, const double* d_u, const double* d_p) {
    H.launches_at_build = H.kernel_launches;
    int rc = build_operator(H, precision, prev, d_u, d_p);
    if (rc != GG_OK) return rc;
    // moments (1 or 2 builds) + K u_b + RHS finish + Gᵀ u_b + negate
    H.kernel_launches += (precision == GG_PRECISION_MIXED ? 2 : 1) + 4;
    // RHS: f_f −= K_fb u_b ; h = −G_bᵀ u_b
    H.ub.ensure(sizeof(double) * H.ndof);
    GG_CUDA(cudaMemsetAsync(H.ub.p, 0, sizeof(double) * H.ndof, H.stream));
    apply_K<double>(H.mk, H.mom64.as<double>(), H.bcmask.as<uint8_t>(), H.bcval.as<double>(), H.ub.as<double>(),
                    H.stream);
    k_finish_rhs<<<grid(H.ndof), 256, 0, H.stream>>>(H.ndof, H.nnode, H.bcmask.as<uint8_t>(), H.ub.as<double>(),
                                                      H.f.as<double>());
    apply_GT(H, H.bcval.as<double>(), H.hvec.as<double>(), H.stream);
    k_neg<<<grid(H.nel), 256, 0, H.stream>>>(H.nel, H.hvec.as<double>());
    GG_CUDA(cudaGetLastError());
    GG_CUDA(cudaStreamSynchronize(H.stream));
    H.built = true;
    H.built_precision = precision;
    H.build_gen++;
    return GG_OK;
}
}  // namespace gg

extern "C" {

int gg_build_operator(gg_handle* h, int32_t precision, int32_t prev, const double* u, const double* p) {
    if (!h) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.located) return gg::set_error(H, GG_ERR_STATE, "gg_locate has not succeeded");
    if (H.n_materials == 0) return gg::set_error(H, GG_ERR_STATE, "materials not set");
    if (H.max_material >= H.n_materials)
        return gg::set_error(H, GG_ERR_INVALID, "a point refers to a material that is not set");
    if (precision != GG_PRECISION_FP64 && precision != GG_PRECISION_MIXED)
        return gg::set_error(H, GG_ERR_INVALID, "precision");
    if (prev && !u) return gg::set_error(H, GG_ERR_INVALID, "previous velocity required");
    int rc = GG_OK;
    GG_TRY(h, {
        const double *du = nullptr, *dp = nullptr;
        if (prev) {
            gg::upload_nodal(H, u, H.prev_u, false);
            du = H.prev_u.as<double>();
            if (p) {
                H.prev_p.ensure(sizeof(double) * H.nel);
                GG_CUDA(cudaMemcpyAsync(H.prev_p.p, p, sizeof(double) * H.nel, cudaMemcpyHostToDevice, H.stream));
                dp = H.prev_p.as<double>();
            }
        }
        rc = gg::build_all(H, precision, prev, du, dp);
    })
    if (rc == GG_ERR_EMPTY_CELL) gg::set_error(H, rc, "an element holds no material point");
    return rc;
}

int gg_uzawa_solve(gg_handle* h, const gg_uzawa_params* prm, double* u, double* p, gg_uzawa_stats* stats) {
    if (!h || !prm || !u || !p) return GG_ERR_INVALID;
    Handle& H = h->H;
    if (!H.built) return gg::set_error(H, GG_ERR_STATE, "operator not built");
    if (prm->precision == GG_PRECISION_MIXED && H.built_precision != GG_PRECISION_MIXED)
        return gg::set_error(H, GG_ERR_STATE, "operator built without the FP32 moments");
    if (!(prm->tolerance > 0) || prm->max_iterations < 1) return gg::set_error(H, GG_ERR_INVALID, "tolerance/iterations");
    int rc = GG_OK;
    gg_uzawa_stats S{};
    GG_TRY(h, {
        if (prm->reuse_pressure)
            GG_CUDA(cudaMemcpyAsync(H.q.p, p, sizeof(double) * H.nel, cudaMemcpyHostToDevice, H.stream));
        else
            GG_CUDA(cudaMemsetAsync(H.q.p, 0, sizeof(double) * H.nel, H.stream));
        rc = gg::uzawa_solve(H, *prm, S);
        gg::store_solution(H);
        gg::download_nodal(H, H.u.as<double>(), H.bcval.as<double>(), u);
        GG_CUDA(cudaMemcpyAsync(p, H.q.p, sizeof(double) * H.nel, cudaMemcpyDeviceToHost, H.stream));
        GG_CUDA(cudaStreamSynchronize(H.stream));
        H.have_solution = true;
    })
    if (stats) *stats = S;
    if (rc != GG_OK)
        gg::set_error(H, rc, "Uzawa solve failed (status " + std::to_string(rc) + ")" +
                                 (H.fail_where.empty() ? std::string() : ": " + H.fail_where));
    return rc;
}

}  // extern "C"
