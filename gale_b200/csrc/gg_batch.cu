// gg_batch.cu -- many independent Stokes problems at once (the uneven batched sweep).
//
// Gale solves one problem per run (one SLE per MPI job).  Here a batch of independent
// problems of different mesh sizes is driven from a shared work queue.
//   * Mixed precision with the multigrid inner solve (the sweep's configuration): `workers`
//     host threads locate and build every problem on its own stream, then ONE launch of the
//     batched CTA solver (gg_cta.cu) runs every Uzawa solve, one problem per CTA, the CTAs
//     pulling problem indices from a device work queue, largest problems first.
//   * Otherwise `workers` host threads pull problem indices from an atomic counter and run
//     locate → build → Uzawa on each handle; every handle owns its stream and CUDA graphs,
//     so the small kernels of different problems overlap on the GPU's 148 SMs.
// GALE_B200_BATCH_CTA=0 selects the second form for any parameters.
#include <atomic>
#include <cstdlib>
#include <string>
#include <cstring>
#include <thread>
#include <vector>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"

namespace gg {
int build_all(Handle& H, int precision, int prev, const double* d_u, const double* d_p);
void store_solution(Handle& H);
}  // namespace gg

namespace {

int solve_one(gg_handle* h, const gg_uzawa_params* prm, double* u, double* p, gg_uzawa_stats* st) {
    // share the GPU with the other problems of the batch; a later lone solve gets the
    // handle's own setting back
    const int keep = h->H.fused_dofs_per_block;
    h->H.fused_dofs_per_block = 1024;
    int rc = gg_locate(h, nullptr);
    if (rc == GG_OK) rc = gg_build_operator(h, prm->precision, 0, nullptr, nullptr);
    if (rc == GG_OK) rc = gg_uzawa_solve(h, prm, u, p, st);
    h->H.fused_dofs_per_block = keep;
    return rc;
}

}  // namespace

static bool batch_cta_enabled() {
    const char* e = getenv("GALE_B200_BATCH_CTA");
    return !(e && e[0] == '0');
}

extern "C" int gg_solve_batch(int32_t n, gg_handle* const* handles, const gg_uzawa_params* params,
                              int32_t workers, double* const* u_out, double* const* p_out,
                              gg_uzawa_stats* stats, int32_t* status) {
    if (n < 1 || !handles || !params || !u_out || !p_out || !status) return GG_ERR_INVALID;
    for (int i = 0; i < n; i++)
        if (!handles[i] || !u_out[i] || !p_out[i]) return GG_ERR_INVALID;
    if (workers < 1) workers = 1;
    if (workers > n) workers = n;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GG_ERR_NO_DEVICE;
    bool cta = batch_cta_enabled() && gg::cta_batch_supported(*params);
    for (int i = 1; i < n && cta; i++)
        if (handles[i]->H.dim != handles[0]->H.dim) cta = false;
    if (cta) {
        // locate and build on the handles' streams, then one launch for every solve
        std::atomic<int> next(0);
        auto prep = [&]() {
            cudaSetDevice(dev);
            for (;;) {
                const int i = next.fetch_add(1);
                if (i >= n) break;
                int rc = gg_locate(handles[i], nullptr);
                if (rc == GG_OK) rc = gg_build_operator(handles[i], params->precision, 0, nullptr, nullptr);
                status[i] = rc;
            }
        };
        std::vector<std::thread> pool;
        for (int w = 1; w < workers; w++) pool.emplace_back(prep);
        prep();
        for (auto& t : pool) t.join();
        for (int i = 0; i < n; i++)
            if (status[i] != GG_OK) return status[i];
        std::vector<gg::Handle*> hs(n);
        for (int i = 0; i < n; i++) hs[i] = &handles[i]->H;
        const int rc = gg::cta_batch_solve(hs, *params, u_out, p_out, stats, status);
        if (rc != GG_OK) return rc;
        for (int i = 0; i < n; i++)
            if (status[i] != GG_OK) {
                gg::set_error(handles[i]->H, status[i], "batched Uzawa solve failed (status " +
                                                            std::to_string(status[i]) + ")");
                return status[i];
            }
        return GG_OK;
    }
    std::atomic<int> next(0);
    auto work = [&]() {
        cudaSetDevice(dev);
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            gg_uzawa_stats st;
            std::memset(&st, 0, sizeof st);
            status[i] = solve_one(handles[i], params, u_out[i], p_out[i], &st);
            if (stats) stats[i] = st;
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < workers; w++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (int i = 0; i < n; i++)
        if (status[i] != GG_OK) return status[i];
    return GG_OK;
}
