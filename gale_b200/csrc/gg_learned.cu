// gg_learned.cu -- learned coarse correction for the inner velocity solve (no counterpart
// in the reference).
//
// A two-layer convolutional network over the nodal grid of one multigrid level L
// (3^dim stencils, 32 hidden channels, BF16 weights, FP32 accumulation):
//     input  x = [ normalised log10 η (node average of the level-L element viscosity),
//                  r_L / s ]                                  (1 + dim channels)
//     h = relu(conv1(x) + b1),  y = conv2(h) + b2,  e_L = s · y   (dim channels)
// where r_L is the fine residual restricted to level L and s its RMS.  In the inner
// flexible CG the preconditioner becomes z = V(r) + P_{0←L} e_L: the network predicts the
// part of the error that one V-cycle leaves, e − V(r), at coarse resolution.
//
// Training data come from the solver itself: on the current operator, for a few right-
// hand sides b (the force vector and G s for random pressures s) the MG solve gives x*;
// a stationary MG iteration x_{k+1} = x_k + V(b − A x_k) then yields pairs
// (r_k = b − A x_k, t_k = x* − x_k − V(r_k)), restricted / injected to level L.
// Forward, backward (data and weight gradients), loss and Adam are hand-written kernels
// below; tests/test_learned.py checks the gradients against oracle/learned_ref.py.
#include <cuda_bf16.h>
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"
#include "gg_ops.cuh"

namespace gg {

namespace {

constexpr int kHidden = 32;

struct NetShape {
    int dim, cin, cout, taps;
    int64_t n1w, n1b, n2w, n2b;  // parameter counts
    int64_t total() const { return n1w + n1b + n2w + n2b; }
};

NetShape net_shape(int dim) {
    NetShape s;
    s.dim = dim;
    s.cin = 1 + dim;
    s.cout = dim;
    s.taps = dim == 3 ? 27 : 9;
    s.n1w = (int64_t)kHidden * s.taps * s.cin;
    s.n1b = kHidden;
    s.n2w = (int64_t)s.cout * s.taps * kHidden;
    s.n2b = s.cout;
    return s;
}

struct Grid3 {
    int nx, ny, nz;
    __host__ __device__ int64_t n() const { return (int64_t)nx * ny * nz; }
};

__device__ __forceinline__ int64_t nbr(const Grid3& g, int64_t n, int t, int dim, bool& ok) {
    const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = dim == 3 ? t / 9 - 1 : 0;
    const int x = (int)(n % g.nx);
    const int64_t r = n / g.nx;
    const int y = (int)(r % g.ny), z = (int)(r / g.ny);
    const int X = x + dx, Y = y + dy, Z = z + dz;
    ok = X >= 0 && Y >= 0 && Z >= 0 && X < g.nx && Y < g.ny && Z < g.nz;
    return X + (int64_t)g.nx * (Y + (int64_t)g.ny * Z);
}

// out[b][o][n] = bias[o] + Σ_t Σ_c W[o][t][c] · x[b][c][n + d_t]   (optional relu; pre-activation kept)
__global__ void k_conv_fwd(Grid3 g, int dim, int B, int cin, int cout, int taps, const float* __restrict__ x,
                           const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias,
                           float* __restrict__ out, float* __restrict__ pre, int relu,
                           const int32_t* __restrict__ done) {
    if (done && *done) return;
    const int64_t N = g.n();
    const int64_t total = (int64_t)B * cout * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = idx % N;
        const int o = (int)((idx / N) % cout);
        const int b = (int)(idx / (N * cout));
        float acc = bias[o];
        for (int t = 0; t < taps; t++) {
            bool ok;
            const int64_t m = nbr(g, n, t, dim, ok);
            if (!ok) continue;
            const __nv_bfloat16* w = W + ((int64_t)o * taps + t) * cin;
            const float* xb = x + (int64_t)b * cin * N + m;
            for (int c = 0; c < cin; c++) acc += __bfloat162float(w[c]) * xb[(int64_t)c * N];
        }
        if (pre) pre[idx] = acc;
        out[idx] = relu ? fmaxf(acc, 0.f) : acc;
    }
}

// din[b][c][n] = Σ_t Σ_o W[o][t][c] · dout[b][o][n − d_t], times 1(pre > 0) when pre is given
__global__ void k_conv_bwd_data(Grid3 g, int dim, int B, int cin, int cout, int taps, const float* __restrict__ dout,
                                const __nv_bfloat16* __restrict__ W, const float* __restrict__ pre,
                                float* __restrict__ din) {
    const int64_t N = g.n();
    const int64_t total = (int64_t)B * cin * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = idx % N;
        const int c = (int)((idx / N) % cin);
        const int b = (int)(idx / (N * cin));
        float acc = 0.f;
        for (int t = 0; t < taps; t++) {
            bool ok;
            const int64_t m = nbr(g, n, taps - 1 - t, dim, ok);  // n − d_t
            if (!ok) continue;
            for (int o = 0; o < cout; o++)
                acc += __bfloat162float(W[((int64_t)o * taps + t) * cin + c]) * dout[((int64_t)b * cout + o) * N + m];
        }
        if (pre && !(pre[idx] > 0.f)) acc = 0.f;
        din[idx] = acc;
    }
}

// dW[o][t][c] = Σ_b Σ_n dout[b][o][n] · x[b][c][n + d_t];  db[o] = Σ dout  (one block per weight)
__global__ void k_conv_bwd_weight(Grid3 g, int dim, int B, int cin, int cout, int taps, const float* __restrict__ dout,
                                  const float* __restrict__ x, float* __restrict__ dW, float* __restrict__ db) {
    const int64_t N = g.n();
    const int64_t nw = (int64_t)cout * taps * cin;
    for (int64_t w = blockIdx.x; w < nw + cout; w += gridDim.x) {
        double acc = 0.0;
        if (w < nw) {
            const int c = (int)(w % cin), t = (int)((w / cin) % taps), o = (int)(w / ((int64_t)cin * taps));
            for (int64_t i = threadIdx.x; i < (int64_t)B * N; i += blockDim.x) {
                const int b = (int)(i / N);
                const int64_t n = i % N;
                bool ok;
                const int64_t m = nbr(g, n, t, dim, ok);
                if (ok) acc += (double)dout[((int64_t)b * cout + o) * N + n] * x[((int64_t)b * cin + c) * N + m];
            }
        } else {
            const int o = (int)(w - nw);
            for (int64_t i = threadIdx.x; i < (int64_t)B * N; i += blockDim.x) {
                const int b = (int)(i / N);
                acc += dout[((int64_t)b * cout + o) * N + (i % N)];
            }
        }
        acc = block_sum(acc);
        if (threadIdx.x == 0) {
            if (w < nw) dW[w] = (float)acc; else db[w - nw] = (float)acc;
        }
        __syncthreads();
    }
}

// dy = 2 w_b m (y − t), per-sample loss partials; w_b = 1/‖m t_b‖²
__global__ void k_loss_grad(int64_t N, int B, int cout, int64_t nnode_lvl, const uint8_t* __restrict__ bc,
                            const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ wgt,
                            float* __restrict__ dy, double* __restrict__ part) {
    double acc = 0.0;
    const int64_t total = (int64_t)B * cout * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = idx % N;
        const int c = (int)((idx / N) % cout);
        const int b = (int)(idx / (N * cout));
        const bool fixed = (bc[n] >> c) & 1;
        const float r = fixed ? 0.f : (y[idx] - t[idx]);
        dy[idx] = 2.f * wgt[b] * r;
        acc += (double)wgt[b] * (double)r * r;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
    (void)nnode_lvl;
}

__global__ void k_adam(int64_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float c1, float c2,
                       __nv_bfloat16* __restrict__ wb) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
        w[i] = wi;
        wb[i] = __float2bfloat16(wi);
    }
}

__global__ void k_to_bf16(int64_t n, const float* __restrict__ a, __nv_bfloat16* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = __float2bfloat16(a[i]);
}

// level-L node field of log10 η: element mean viscosity M_1/vol, averaged over adjacent elements
template <int DIM>
__global__ void k_logeta_nodes(MeshK mk, const double* __restrict__ mom, double vol, float* __restrict__ out) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < mk.nnode; n += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(n % mk.nn[0]);
        const int64_t rr = n / mk.nn[0];
        const int j = (int)(rr % mk.nn[1]), k = DIM == 3 ? (int)(rr / mk.nn[1]) : 0;
        double s = 0.0;
        int cnt = 0;
        for (int a = 0; a < (1 << DIM); a++) {
            const int ei = i - (a & 1), ej = j - ((a >> 1) & 1), ek = DIM == 3 ? k - ((a >> 2) & 1) : 0;
            if (ei < 0 || ej < 0 || ek < 0 || ei >= mk.n[0] || ej >= mk.n[1] || ek >= mk.n[2]) continue;
            const int64_t e = ei + (int64_t)mk.n[0] * (ej + (int64_t)mk.n[1] * ek);
            s += log10(fmax(mom[e] / vol, 1e-300));
            cnt++;
        }
        out[n] = (float)(s / cnt);
    }
}

// standardise a field in place (single block)
__global__ void k_standardise(int64_t n, float* __restrict__ a) {
    double s = 0.0, s2 = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) { s += a[i]; s2 += (double)a[i] * a[i]; }
    s = block_sum(s);
    __syncthreads();
    s2 = block_sum(s2);
    __shared__ float mu, sd;
    if (threadIdx.x == 0) {
        mu = (float)(s / n);
        const double var = s2 / n - (s / n) * (s / n);
        sd = (float)(var > 1e-12 ? sqrt(var) : 1.0);
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) a[i] = (a[i] - mu) / sd;
}

// network input [1+dim][N] from the level-L residual: scale s = RMS(r_L) stored in *scale
__global__ void k_nn_input(int64_t N, int dim, const float* __restrict__ logeta, const float* __restrict__ rL,
                           float* __restrict__ xin, float* __restrict__ scale, const int32_t* __restrict__ done) {
    if (done && *done) return;
    double s2 = 0.0;
    for (int64_t i = threadIdx.x; i < N * dim; i += blockDim.x) s2 += (double)rL[i] * rL[i];
    s2 = block_sum(s2);
    __shared__ float inv;
    if (threadIdx.x == 0) {
        const float s = (float)sqrt(s2 / (double)(N * dim));
        *scale = s;
        inv = s > 0.f ? 1.f / s : 0.f;
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) xin[i] = logeta[i];
    for (int64_t i = threadIdx.x; i < N * dim; i += blockDim.x) xin[N + i] = rL[i] * inv;
}

// e_L = s·y on free dofs
__global__ void k_nn_output(int64_t N, int dim, const uint8_t* __restrict__ bc, const float* __restrict__ y,
                            const float* __restrict__ scale, float* __restrict__ eL, const int32_t* __restrict__ done) {
    if (done && *done) return;
    const float s = *scale;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N * dim; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i / N);
        eL[i] = ((bc[i - (int64_t)c * N] >> c) & 1) ? 0.f : s * y[i];
    }
}

__global__ void k_resid_after(int64_t n, const float* __restrict__ r, const float* __restrict__ t,
                              float* __restrict__ out, const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = r[i] - t[i];
}

__global__ void k_zero(int64_t n, float* __restrict__ a, const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) a[i] = 0.f;
}

int g(int64_t n) { return grid_for(n, 256); }

constexpr int kOmegaBlocks = 296;

// ω = max(0, (d·r')/(dᵀA d)): the step along the learned direction d that minimises the
// energy norm of the error left after z + ω d (r' = r − A z).  Per-block partials, the
// last block to arrive sums them in block order; layout of w: [2·blocks partials][ω][pad]
// then the arrival counter.
__global__ void k_omega(int64_t n, const float* __restrict__ d, const float* __restrict__ r1,
                        const float* __restrict__ ad, double* __restrict__ w, const int32_t* __restrict__ done) {
    if (done && *done) return;
    double num = 0.0, den = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        num += (double)d[i] * (double)r1[i];
        den += (double)d[i] * (double)ad[i];
    }
    __shared__ double s_num[32], s_den[32];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) {
        num += __shfl_down_sync(0xffffffffu, num, o);
        den += __shfl_down_sync(0xffffffffu, den, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        s_num[wid] = num;
        s_den[wid] = den;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            a += s_num[k];
            b += s_den[k];
        }
        w[2 * blockIdx.x] = a;
        w[2 * blockIdx.x + 1] = b;
        __threadfence();
        unsigned int* counter = reinterpret_cast<unsigned int*>(w + 2 * gridDim.x + 2);
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double a = 0.0, b = 0.0;
    for (int k = 0; k < (int)gridDim.x; k++) {
        a += w[2 * k];
        b += w[2 * k + 1];
    }
    w[2 * gridDim.x] = (b > 0.0 && a > 0.0) ? a / b : 0.0;
    *reinterpret_cast<unsigned int*>(w + 2 * gridDim.x + 2) = 0u;
}

// z += ω d with ω from k_omega
__global__ void k_axpy_omega(int64_t n, const double* __restrict__ omega, const float* __restrict__ d,
                             float* __restrict__ z, const int32_t* __restrict__ done) {
    if (done && *done) return;
    const float w = (float)*omega;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        z[i] += w * d[i];
}

}  // namespace

// restriction / prolongation kernels of gg_mg.cu
void mg_restrict(Handle& H, size_t l, const float* fine, float* coarse, const int32_t* done);
void mg_prolong_add(Handle& H, size_t l, const float* coarse, float* fine, const int32_t* done);

struct LearnedState {
    NetShape shape{};
    Grid3 grid{};
    size_t level = 0;
    DBuf w32, wbf, grad, adam_m, adam_v;  // master weights, BF16 copy, grads, Adam moments
    DBuf logeta;                          // standardised level-L log10 η [N]
    std::vector<std::unique_ptr<DBuf>> rl, el;  // per-level restricted residual / correction
    DBuf xin, h, pre, y, scale;                 // inference buffers (batch 1)
    DBuf t0, r0;                                // fine-level A z and r − A z
    int64_t gen = -1;                           // build generation of logeta
    int base = GG_LEARN_BASE_MULTIGRID;         // preconditioner the weights correct
    DBuf d0, ad0, wred;                         // fine correction d, A d, ω reduction scratch
};

LearnedState& learned(Handle& H) {
    if (!H.learned) H.learned = std::make_shared<LearnedState>();
    return *H.learned;
}

static void ensure_net(Handle& H, size_t level) {
    LearnedState& S = learned(H);
    const int dim = H.dim;
    S.shape = net_shape(dim);
    S.level = level;
    const MeshK& mk = H.mg[level]->mk;
    S.grid = Grid3{mk.nn[0], mk.nn[1], mk.nn[2]};
    const int64_t P = S.shape.total();
    S.w32.ensure(sizeof(float) * P);
    S.wbf.ensure(sizeof(__nv_bfloat16) * P);
    S.grad.ensure(sizeof(float) * P);
    S.adam_m.ensure(sizeof(float) * P);
    S.adam_v.ensure(sizeof(float) * P);
    const int64_t N = S.grid.n();
    S.logeta.ensure(sizeof(float) * N);
    S.xin.ensure(sizeof(float) * (1 + dim) * N);
    S.h.ensure(sizeof(float) * kHidden * N);
    S.pre.ensure(sizeof(float) * kHidden * N);
    S.y.ensure(sizeof(float) * dim * N);
    S.scale.ensure(sizeof(float) * 4);
    S.t0.ensure(sizeof(float) * H.ndof);
    S.r0.ensure(sizeof(float) * H.ndof);
    S.d0.ensure(sizeof(float) * H.ndof);
    S.ad0.ensure(sizeof(float) * H.ndof);
    S.wred.ensure(sizeof(double) * (2 * kOmegaBlocks + 2) + 16);
    GG_CUDA(cudaMemsetAsync(S.wred.p, 0, sizeof(double) * (2 * kOmegaBlocks + 2) + 16, H.stream));
    if (S.rl.size() != level + 1) {
        S.rl.clear();
        S.el.clear();
        for (size_t l = 0; l <= level; l++) {
            S.rl.push_back(std::make_unique<DBuf>());
            S.el.push_back(std::make_unique<DBuf>());
            S.rl.back()->ensure(sizeof(float) * H.mg[l]->ndof);
            S.el.back()->ensure(sizeof(float) * H.mg[l]->ndof);
        }
    }
}

// Refresh the level-L viscosity input for the current operator build.
static void learned_refresh(Handle& H) {
    LearnedState& S = learned(H);
    if (S.gen == H.build_gen) return;
    MGLevel& L = *H.mg[S.level];
    double vol = 1.0;
    for (int d = 0; d < H.dim; d++) vol *= L.mk.h[d];
    if (H.dim == 2) k_logeta_nodes<2><<<g(L.nnode), 256, 0, H.stream>>>(L.mk, L.mom64, vol, S.logeta.as<float>());
    else k_logeta_nodes<3><<<g(L.nnode), 256, 0, H.stream>>>(L.mk, L.mom64, vol, S.logeta.as<float>());
    k_standardise<<<1, 1024, 0, H.stream>>>(L.nnode, S.logeta.as<float>());
    GG_CUDA(cudaGetLastError());
    H.kernel_launches += 2;
    S.gen = H.build_gen;
}

static void net_forward(Handle& H, int B, const float* xin, float* hbuf, float* pre, float* y, const int32_t* done) {
    LearnedState& S = learned(H);
    const NetShape& sh = S.shape;
    const int64_t N = S.grid.n();
    const __nv_bfloat16* W1 = S.wbf.as<__nv_bfloat16>();
    const float* b1 = S.w32.as<float>() + sh.n1w;  // biases stay FP32
    const __nv_bfloat16* W2 = W1 + sh.n1w + sh.n1b;
    const float* b2 = S.w32.as<float>() + sh.n1w + sh.n1b + sh.n2w;
    k_conv_fwd<<<g((int64_t)B * kHidden * N), 256, 0, H.stream>>>(S.grid, H.dim, B, sh.cin, kHidden, sh.taps, xin, W1, b1,
                                                                  hbuf, pre, 1, done);
    k_conv_fwd<<<g((int64_t)B * sh.cout * N), 256, 0, H.stream>>>(S.grid, H.dim, B, kHidden, sh.cout, sh.taps, hbuf, W2,
                                                                  b2, y, nullptr, 0, done);
    H.kernel_launches += 2;
}

// z += ω P_{0←L} N(R_{L←0} r'), r' = r − A z: enqueued inside the captured inner iteration
void learned_correction(Handle& H, const float* r, float* z, const int32_t* done) {
    LearnedState& S = learned(H);
    const size_t Lv = S.level;
    const int dim = H.dim;
    // residual the V-cycle leaves: r' = r − A z
    MGLevel& L0 = *H.mg[0];
    k_zero<<<g(H.ndof), 256, 0, H.stream>>>(H.ndof, S.t0.as<float>(), done);
    apply_K_ex<float>(L0.mk, L0.mom32, L0.bcmask, z, S.t0.as<float>(), nullptr, apply_grid(L0.nel), H.stream, done);
    k_resid_after<<<g(H.ndof), 256, 0, H.stream>>>(H.ndof, r, S.t0.as<float>(), S.r0.as<float>(), done);
    H.kernel_launches += 3;
    const float* src = S.r0.as<float>();
    for (size_t l = 1; l <= Lv; l++) {
        mg_restrict(H, l, src, S.rl[l]->as<float>(), done);
        src = S.rl[l]->as<float>();
    }
    const int64_t N = S.grid.n();
    k_nn_input<<<1, 1024, 0, H.stream>>>(N, dim, S.logeta.as<float>(), src, S.xin.as<float>(), S.scale.as<float>(), done);
    net_forward(H, 1, S.xin.as<float>(), S.h.as<float>(), nullptr, S.y.as<float>(), done);
    k_nn_output<<<g(N * dim), 256, 0, H.stream>>>(N, dim, H.mg[Lv]->bcmask, S.y.as<float>(), S.scale.as<float>(),
                                                  S.el[Lv]->as<float>(), done);
    H.kernel_launches += 2;
    // d = P_{0←L} N(·) on the fine level
    for (size_t l = Lv; l >= 1; l--) {
        float* dst = (l == 1) ? S.d0.as<float>() : S.el[l - 1]->as<float>();
        k_zero<<<g(H.mg[l - 1]->ndof), 256, 0, H.stream>>>(H.mg[l - 1]->ndof, dst, done);
        H.kernel_launches++;
        mg_prolong_add(H, l, S.el[l]->as<float>(), dst, done);
    }
    // z += ω d with the energy-optimal ω ≥ 0, so the correction never raises the error
    k_zero<<<g(H.ndof), 256, 0, H.stream>>>(H.ndof, S.ad0.as<float>(), done);
    apply_K_ex<float>(L0.mk, L0.mom32, L0.bcmask, S.d0.as<float>(), S.ad0.as<float>(), nullptr, apply_grid(L0.nel),
                      H.stream, done);
    k_omega<<<kOmegaBlocks, 256, 0, H.stream>>>(H.ndof, S.d0.as<float>(), S.r0.as<float>(), S.ad0.as<float>(),
                                                 S.wred.as<double>(), done);
    k_axpy_omega<<<g(H.ndof), 256, 0, H.stream>>>(H.ndof, S.wred.as<double>() + 2 * kOmegaBlocks,
                                                  S.d0.as<float>(), z, done);
    H.kernel_launches += 4;
}

bool learned_ready(Handle& H) { return H.learned && H.nn_ready; }

int learned_base(Handle& H) { return H.learned ? H.learned->base : -1; }

namespace {
// z = D⁻¹ r on the fine level (FP32 Jacobi diagonal, zero on BC rows)
__global__ void k_jacobi_z(int64_t n, const float* __restrict__ invd, const float* __restrict__ r,
                           float* __restrict__ z, const int32_t* __restrict__ done) {
    if (done && *done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        z[i] = invd[i] * r[i];
}
// x += ω z
__global__ void k_axpyw(int64_t n, float w, const float* __restrict__ z, float* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += w * z[i];
}
}  // namespace

// z = D⁻¹ r: the plain Jacobi preconditioner, enqueued inside captured iterations
void jacobi_precond(Handle& H, const float* r, float* z, const int32_t* done) {
    const MGLevel& L0 = *H.mg[0];
    k_jacobi_z<<<g(H.ndof), 256, 0, H.stream>>>(H.ndof, L0.invdiag.as<float>(), r, z, done);
    H.kernel_launches++;
}

void learned_prepare(Handle& H) {
    if (!learned_ready(H)) return;
    learned_refresh(H);
}

// ---------------------------------------------------------------- training ----
namespace {
__global__ void k_cast_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}
__global__ void k_sub(int64_t n, const float* __restrict__ b, const float* __restrict__ t, float* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - t[i];
}
__global__ void k_target(int64_t n, const float* __restrict__ xs, const float* __restrict__ xk,
                         const float* __restrict__ zk, float* __restrict__ t) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        t[i] = xs[i] - xk[i] - zk[i];
}
__global__ void k_axpy1(int64_t n, const float* __restrict__ z, float* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += z[i];
}
// target at level L: the fine error at the level-L node positions, divided by the input scale
__global__ void k_inject(MeshK fk, MeshK ck, int stride, int dim, const float* __restrict__ tf,
                         float* __restrict__ out, const float* __restrict__ scale) {
    const float s = *scale;
    const float inv = s > 0.f ? 1.f / s : 0.f;
    for (int64_t N = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; N < ck.nnode; N += (int64_t)gridDim.x * blockDim.x) {
        const int I = (int)(N % ck.nn[0]);
        const int64_t rr = N / ck.nn[0];
        const int J = (int)(rr % ck.nn[1]), K = (int)(rr / ck.nn[1]);
        const int64_t n = (int64_t)stride * I + (int64_t)fk.nn[0] * ((int64_t)stride * J + (int64_t)fk.nn[1] * stride * K);
        for (int c = 0; c < dim; c++) out[(int64_t)c * ck.nnode + N] = tf[(int64_t)c * fk.nnode + n] * inv;
    }
}
}  // namespace

static void train_cast(Handle& H, const double* a, float* b, int64_t n) {
    k_cast_f32<<<g(n), 256, 0, H.stream>>>(n, a, b);
}
static void train_residual(Handle& H, const float* b, const float* x, float* r) {
    MGLevel& L0 = *H.mg[0];
    float* t = H.mg_xt.as<float>();
    GG_CUDA(cudaMemsetAsync(t, 0, sizeof(float) * H.ndof, H.stream));
    apply_K_ex<float>(L0.mk, L0.mom32, L0.bcmask, x, t, nullptr, apply_grid(L0.nel), H.stream, nullptr);
    k_sub<<<g(H.ndof), 256, 0, H.stream>>>(H.ndof, b, t, r);
}
static void train_target(Handle& H, const float* xs, const float* xk, const float* zk, float* t) {
    k_target<<<g(H.ndof), 256, 0, H.stream>>>(H.ndof, xs, xk, zk, t);
}
static void train_axpy(Handle& H, const float* z, float* x) { k_axpy1<<<g(H.ndof), 256, 0, H.stream>>>(H.ndof, z, x); }
static void train_inject(Handle& H, size_t level, const float* tf, float* out, const float* scale) {
    const MeshK& ck = H.mg[level]->mk;
    k_inject<<<g(ck.nnode), 256, 0, H.stream>>>(H.mk, ck, 1 << level, H.dim, tf, out, scale);
}

// Forward + loss + backward on a batch already on the device; returns the loss.
static double train_step(Handle& H, int B, const float* xin, const float* tgt, const float* wgt, DBuf& hbuf, DBuf& pre,
                         DBuf& y, DBuf& dy, DBuf& dh, DBuf& part) {
    LearnedState& S = learned(H);
    const NetShape& sh = S.shape;
    const int64_t N = S.grid.n();
    net_forward(H, B, xin, hbuf.as<float>(), pre.as<float>(), y.as<float>(), nullptr);
    const int nbl = 64;
    k_loss_grad<<<nbl, 256, 0, H.stream>>>(N, B, sh.cout, N, H.mg[S.level]->bcmask, y.as<float>(), tgt, wgt,
                                           dy.as<float>(), part.as<double>());
    float* G = S.grad.as<float>();
    const __nv_bfloat16* W2 = S.wbf.as<__nv_bfloat16>() + sh.n1w + sh.n1b;
    k_conv_bwd_weight<<<1024, 256, 0, H.stream>>>(S.grid, H.dim, B, kHidden, sh.cout, sh.taps, dy.as<float>(), hbuf.as<float>(),
                                                  G + sh.n1w + sh.n1b, G + sh.n1w + sh.n1b + sh.n2w);
    k_conv_bwd_data<<<g((int64_t)B * kHidden * N), 256, 0, H.stream>>>(S.grid, H.dim, B, kHidden, sh.cout, sh.taps, dy.as<float>(),
                                                                      W2, pre.as<float>(), dh.as<float>());
    k_conv_bwd_weight<<<1024, 256, 0, H.stream>>>(S.grid, H.dim, B, sh.cin, kHidden, sh.taps, dh.as<float>(), xin, G, G + sh.n1w);
    GG_CUDA(cudaGetLastError());
    std::vector<double> hp(nbl);
    GG_CUDA(cudaMemcpyAsync(hp.data(), part.p, sizeof(double) * nbl, cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
    double loss = 0.0;
    for (double v : hp) loss += v;
    return loss;
}

static void init_weights(Handle& H, uint64_t seed) {
    LearnedState& S = learned(H);
    const NetShape& sh = S.shape;
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<float> w(sh.total(), 0.f);
    const double s1 = sqrt(2.0 / (sh.taps * sh.cin)), s2 = 0.1 * sqrt(1.0 / (sh.taps * kHidden));
    for (int64_t i = 0; i < sh.n1w; i++) w[i] = (float)(s1 * nd(rng));
    for (int64_t i = 0; i < sh.n2w; i++) w[sh.n1w + sh.n1b + i] = (float)(s2 * nd(rng));
    GG_CUDA(cudaMemcpyAsync(S.w32.p, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, H.stream));
    k_to_bf16<<<g(sh.total()), 256, 0, H.stream>>>(sh.total(), S.w32.as<float>(), S.wbf.as<__nv_bfloat16>());
    GG_CUDA(cudaMemsetAsync(S.adam_m.p, 0, sizeof(float) * sh.total(), H.stream));
    GG_CUDA(cudaMemsetAsync(S.adam_v.p, 0, sizeof(float) * sh.total(), H.stream));
}

int learned_set_level(Handle& H, int level) {
    int rc = mg_setup(H);
    if (rc != GG_OK) return rc;
    if (H.mg.size() < 2) return set_error(H, GG_ERR_INVALID, "the multigrid hierarchy has a single level");
    if (level >= (int)H.mg.size())
        return set_error(H, GG_ERR_INVALID, "learned level " + std::to_string(level) + " does not exist (levels 1.." +
                                                std::to_string(H.mg.size() - 1) + ")");
    size_t L = level <= 0 ? std::min<size_t>(2, H.mg.size() - 1) : (size_t)level;
    if (!H.learned || learned(H).level != L || learned(H).w32.p == nullptr) ensure_net(H, L);
    H.nn_level = (int)L;
    return GG_OK;
}

int64_t learned_param_count(Handle& H) { return net_shape(H.dim).total(); }

void learned_set_weights(Handle& H, const float* w) {
    LearnedState& S = learned(H);
    const int64_t P = S.shape.total();
    GG_CUDA(cudaMemcpyAsync(S.w32.p, w, sizeof(float) * P, cudaMemcpyHostToDevice, H.stream));
    k_to_bf16<<<g(P), 256, 0, H.stream>>>(P, S.w32.as<float>(), S.wbf.as<__nv_bfloat16>());
    GG_CUDA(cudaStreamSynchronize(H.stream));
    H.nn_ready = true;
    H.nn_verdict = -1;  // new weights: judge again
}

void learned_get_weights(Handle& H, float* w) {
    LearnedState& S = learned(H);
    GG_CUDA(cudaMemcpyAsync(w, S.w32.p, sizeof(float) * S.shape.total(), cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
}

// Forward + backward of a host batch (gradient check): output y, gradient, loss.
int learned_eval(Handle& H, int B, const float* xin_h, const float* tgt_h, const float* w_h, float* y_h, float* grad_h,
                 double* loss) {
    LearnedState& S = learned(H);
    const NetShape& sh = S.shape;
    const int64_t N = S.grid.n();
    learned_set_weights(H, w_h);
    DBuf xin, tgt, wgt, hb, pre, y, dy, dh, part;
    xin.ensure(sizeof(float) * B * sh.cin * N);
    tgt.ensure(sizeof(float) * B * sh.cout * N);
    wgt.ensure(sizeof(float) * B);
    hb.ensure(sizeof(float) * B * kHidden * N);
    pre.ensure(sizeof(float) * B * kHidden * N);
    y.ensure(sizeof(float) * B * sh.cout * N);
    dy.ensure(sizeof(float) * B * sh.cout * N);
    dh.ensure(sizeof(float) * B * kHidden * N);
    part.ensure(sizeof(double) * 64);
    GG_CUDA(cudaMemcpyAsync(xin.p, xin_h, sizeof(float) * B * sh.cin * N, cudaMemcpyHostToDevice, H.stream));
    GG_CUDA(cudaMemcpyAsync(tgt.p, tgt_h, sizeof(float) * B * sh.cout * N, cudaMemcpyHostToDevice, H.stream));
    // per-sample weights 1/‖m t‖² on the host
    std::vector<uint8_t> bc(N);
    GG_CUDA(cudaMemcpyAsync(bc.data(), H.mg[S.level]->bcmask, N, cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
    std::vector<float> w(B);
    for (int b = 0; b < B; b++) {
        double s = 0.0;
        for (int c = 0; c < sh.cout; c++)
            for (int64_t n = 0; n < N; n++)
                if (!((bc[n] >> c) & 1)) {
                    const double t = tgt_h[((int64_t)b * sh.cout + c) * N + n];
                    s += t * t;
                }
        w[b] = (float)(1.0 / (s > 1e-300 ? s : 1e-300));
    }
    GG_CUDA(cudaMemcpyAsync(wgt.p, w.data(), sizeof(float) * B, cudaMemcpyHostToDevice, H.stream));
    *loss = train_step(H, B, xin.as<float>(), tgt.as<float>(), wgt.as<float>(), hb, pre, y, dy, dh, part);
    GG_CUDA(cudaMemcpyAsync(y_h, y.p, sizeof(float) * B * sh.cout * N, cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaMemcpyAsync(grad_h, S.grad.p, sizeof(float) * sh.total(), cudaMemcpyDeviceToHost, H.stream));
    GG_CUDA(cudaStreamSynchronize(H.stream));
    return GG_OK;
}

// Generate (r, e − V(r)) pairs with the solver on the current operator and train.
int learned_train(Handle& H, const gg_learn_params& P, gg_learn_stats& st) {
    std::memset(&st, 0, sizeof st);
    int rc = learned_set_level(H, P.level);
    if (rc != GG_OK) return rc;
    LearnedState& S = learned(H);
    const NetShape& sh = S.shape;
    const int dim = H.dim;
    const int64_t N = S.grid.n();
    const int64_t nd = H.ndof;
    if (P.base != GG_LEARN_BASE_MULTIGRID && P.base != GG_LEARN_BASE_JACOBI)
        return set_error(H, GG_ERR_INVALID, "learned base");
    S.base = P.base;
    const bool jac = S.base == GG_LEARN_BASE_JACOBI;
    // damped Jacobi that advances the sampled iterates: ω = 1/λ_max(D⁻¹A)
    const float omega = (float)(1.0 / H.mg[0]->lambda_max);
    learned_refresh(H);
    GG_CUDA(cudaEventRecord(H.ev0, H.stream));
    init_weights(H, (uint64_t)P.seed * 7919ull + 17ull);
    const int nrhs = P.n_rhs > 0 ? P.n_rhs : 4;
    const int kits = P.iters_per_rhs > 0 ? P.iters_per_rhs : 6;
    const int nsamp = nrhs * kits;
    DBuf X, T, Wt;
    X.ensure(sizeof(float) * nsamp * sh.cin * N);
    T.ensure(sizeof(float) * nsamp * sh.cout * N);
    Wt.ensure(sizeof(float) * nsamp);
    float* b32 = H.r32.as<float>();
    float* xs = H.mg_xs.as<float>();     // x*
    float* xk = H.mg_xk.as<float>();     // stationary iterate
    float* rk = H.cgr32.as<float>();
    float* zk = H.z32.as<float>();
    float* tk = H.p32.as<float>();
    std::mt19937_64 rng((uint64_t)P.seed);
    std::normal_distribution<double> nd01(0.0, 1.0);
    std::vector<double> s_host(H.nel);
    std::vector<float> wts;
    std::vector<uint8_t> bcL(N);
    GG_CUDA(cudaMemcpyAsync(bcL.data(), H.mg[S.level]->bcmask, N, cudaMemcpyDeviceToHost, H.stream));
    int samp = 0;
    std::vector<float> ec;
    for (int j = 0; j < nrhs; j++) {
        if (jac) {
            // Jacobi base: the error a coarse correction must remove lives in the coarse
            // space -- x* = P e_L for a random level-L vector e_L, b = A x*
            const MGLevel& LL = *H.mg[S.level];
            ec.resize((size_t)dim * LL.nnode);
            for (auto& v : ec) v = (float)nd01(rng);
            GG_CUDA(cudaMemcpyAsync(S.el[S.level]->p, ec.data(), sizeof(float) * ec.size(), cudaMemcpyHostToDevice,
                                    H.stream));
            for (size_t l = S.level; l >= 1; l--) {
                float* dst = (l == 1) ? xs : S.el[l - 1]->as<float>();
                GG_CUDA(cudaMemsetAsync(dst, 0, sizeof(float) * (l == 1 ? nd : H.mg[l - 1]->ndof), H.stream));
                mg_prolong_add(H, l, S.el[l]->as<float>(), dst, nullptr);
            }
            GG_CUDA(cudaMemsetAsync(zk, 0, sizeof(float) * nd, H.stream));
            train_residual(H, zk, xs, rk);  // rk = −A x*
            GG_CUDA(cudaMemsetAsync(b32, 0, sizeof(float) * nd, H.stream));
            k_axpyw<<<g(nd), 256, 0, H.stream>>>(nd, -1.f, rk, b32);
        }
        if (!jac) {
            // multigrid base: right-hand sides the solver meets -- the force vector, then
            // G s for random pressures, with x* from the multigrid solve
            if (j == 0) {
                train_cast(H, H.f.as<double>(), b32, nd);
            } else {
                for (auto& v : s_host) v = nd01(rng);
                GG_CUDA(cudaMemcpyAsync(H.qtmp.p, s_host.data(), sizeof(double) * H.nel, cudaMemcpyHostToDevice,
                                        H.stream));
                apply_G(H, H.qtmp.as<double>(), H.ftmp.as<double>(), H.stream);
                train_cast(H, H.ftmp.as<double>(), b32, nd);
            }
            int its = 0;
            rc = fcg_mg_solve(H, b32, xs, 1e-6, 2000, &its);
            if (rc != GG_OK) return rc;
        }
        GG_CUDA(cudaMemsetAsync(xk, 0, sizeof(float) * nd, H.stream));
        for (int k = 0; k < kits; k++) {
            // r = b − A x_k ; z = M(r) (V-cycle or D⁻¹) ; t = x* − x_k − z
            train_residual(H, b32, xk, rk);
            if (jac) jacobi_precond(H, rk, zk, nullptr);
            else vcycle(H, 0, rk, zk, nullptr);
            train_target(H, xs, xk, zk, tk);
            // input: the residual the base preconditioner leaves, r' = r − A z (t = A⁻¹ r');
            // restricted to level L; target t injected to level L
            {
                MGLevel& L0 = *H.mg[0];
                k_zero<<<g(nd), 256, 0, H.stream>>>(nd, S.t0.as<float>(), nullptr);
                apply_K_ex<float>(L0.mk, L0.mom32, L0.bcmask, zk, S.t0.as<float>(), nullptr, apply_grid(L0.nel),
                                  H.stream, nullptr);
                k_resid_after<<<g(nd), 256, 0, H.stream>>>(nd, rk, S.t0.as<float>(), S.r0.as<float>(), nullptr);
            }
            const float* src = S.r0.as<float>();
            for (size_t l = 1; l <= S.level; l++) {
                mg_restrict(H, l, src, S.rl[l]->as<float>(), nullptr);
                src = S.rl[l]->as<float>();
            }
            k_nn_input<<<1, 1024, 0, H.stream>>>(N, dim, S.logeta.as<float>(), src, X.as<float>() + (int64_t)samp * sh.cin * N,
                                                 S.scale.as<float>(), nullptr);
            train_inject(H, S.level, tk, T.as<float>() + (int64_t)samp * sh.cout * N, S.scale.as<float>());
            // per-sample weight
            std::vector<float> th(sh.cout * N);
            GG_CUDA(cudaMemcpyAsync(th.data(), T.as<float>() + (int64_t)samp * sh.cout * N, sizeof(float) * sh.cout * N,
                                    cudaMemcpyDeviceToHost, H.stream));
            GG_CUDA(cudaStreamSynchronize(H.stream));
            double s = 0.0;
            for (int c = 0; c < sh.cout; c++)
                for (int64_t n = 0; n < N; n++)
                    if (!((bcL[n] >> c) & 1)) s += (double)th[c * N + n] * th[c * N + n];
            wts.push_back((float)(1.0 / (s > 1e-30 ? s : 1e-30)));
            samp++;
            if (jac) {
                // the next sample four damped Jacobi steps on: a smoother, larger error
                for (int q = 0; q < 4; q++) {
                    train_residual(H, b32, xk, rk);
                    jacobi_precond(H, rk, zk, nullptr);
                    k_axpyw<<<g(nd), 256, 0, H.stream>>>(nd, omega, zk, xk);
                }
            } else {
                train_axpy(H, zk, xk);  // x_{k+1} = x_k + V(r_k)
            }
        }
    }
    GG_CUDA(cudaMemcpyAsync(Wt.p, wts.data(), sizeof(float) * nsamp, cudaMemcpyHostToDevice, H.stream));
    // Adam over minibatches
    const int B = std::min(8, nsamp);
    DBuf hb, pre, y, dy, dh, part, xb, tb, wb;
    hb.ensure(sizeof(float) * B * kHidden * N);
    pre.ensure(sizeof(float) * B * kHidden * N);
    y.ensure(sizeof(float) * B * sh.cout * N);
    dy.ensure(sizeof(float) * B * sh.cout * N);
    dh.ensure(sizeof(float) * B * kHidden * N);
    part.ensure(sizeof(double) * 64);
    const int epochs = P.epochs > 0 ? P.epochs : 60;
    const float lr = P.lr > 0 ? P.lr : 2e-3f;
    const float b1 = 0.9f, b2 = 0.999f;
    int step = 0;
    double first = -1.0, last = 0.0;
    std::vector<int> order(nsamp);
    for (int i = 0; i < nsamp; i++) order[i] = i;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(order.begin(), order.end(), rng);
        double eloss = 0.0;
        for (int s0 = 0; s0 + B <= nsamp; s0 += B) {
            // contiguous minibatch: gather the chosen samples
            xb.ensure(sizeof(float) * B * sh.cin * N);
            tb.ensure(sizeof(float) * B * sh.cout * N);
            wb.ensure(sizeof(float) * B);
            for (int b = 0; b < B; b++) {
                const int i = order[s0 + b];
                GG_CUDA(cudaMemcpyAsync(xb.as<float>() + (int64_t)b * sh.cin * N, X.as<float>() + (int64_t)i * sh.cin * N,
                                        sizeof(float) * sh.cin * N, cudaMemcpyDeviceToDevice, H.stream));
                GG_CUDA(cudaMemcpyAsync(tb.as<float>() + (int64_t)b * sh.cout * N, T.as<float>() + (int64_t)i * sh.cout * N,
                                        sizeof(float) * sh.cout * N, cudaMemcpyDeviceToDevice, H.stream));
                GG_CUDA(cudaMemcpyAsync(wb.as<float>() + b, Wt.as<float>() + i, sizeof(float), cudaMemcpyDeviceToDevice,
                                        H.stream));
            }
            const double loss = train_step(H, B, xb.as<float>(), tb.as<float>(), wb.as<float>(), hb, pre, y, dy, dh, part);
            eloss += loss / B;
            step++;
            const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
            k_adam<<<g(sh.total()), 256, 0, H.stream>>>(sh.total(), S.w32.as<float>(), S.grad.as<float>(),
                                                         S.adam_m.as<float>(), S.adam_v.as<float>(), lr, b1, b2, c1, c2,
                                                         S.wbf.as<__nv_bfloat16>());
        }
        const double nb = (double)(nsamp / B);
        if (first < 0) first = eloss / nb;
        last = eloss / nb;
    }
    GG_CUDA(cudaEventRecord(H.ev1, H.stream));
    GG_CUDA(cudaEventSynchronize(H.ev1));
    float ms = 0.f;
    GG_CUDA(cudaEventElapsedTime(&ms, H.ev0, H.ev1));
    H.nn_ready = true;
    H.nn_verdict = -1;  // new weights: judge again
    st.samples = nsamp;
    st.loss_first = (float)first;
    st.loss_last = (float)last;
    st.train_ms = ms;
    return GG_OK;
}

}  // namespace gg
