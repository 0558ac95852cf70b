// Batched sweep: many independent GFIEM systems (different grid sizes,
// wavelengths and designs) solved on one GPU.
//
// The reference solves one system per call and synchronises the device after
// every kernel (CUDA_GMRES/launch_GMRES.cuh:88-235 loops over sizes and
// repetitions serially).  Here `nworkers` host threads each own a solver
// context with its own CUDA stream and workspace; they take systems from a
// shared queue ordered largest grid first, so the many small solves of a sweep
// fill the GPU next to the large ones and each context reuses its buffers for
// consecutive systems of the same size.  The operator set-up, the autotuned
// launch shapes (cached per device and embedding size) and the solve are the
// single-system paths; results are per system.  With more than one worker the
// contexts are marked as sharing the GPU, so their autotuner leaves out the
// persistent column pass (one block of ~200 KB shared memory on every SM,
// which would make the other workers' kernels wait).
#include <algorithm>
#include <atomic>
#include <thread>
#include <time.h>
#include <vector>

#include "../../include/cugmres.h"
#include "cg_internal.h"

namespace {

double now_s() {
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

}  // namespace

extern "C" int cugmres_solve_batch(int device, int nsys, const cg_system *sys, const cg_opts *opts, int nworkers,
                                   cg_result *results) {
    if (nsys < 0 || (nsys > 0 && (!sys || !results)) || nworkers < 1) return CG_ERR_INVALID;
    for (int i = 0; i < nsys; i++)
        if (sys[i].N < 1 || !sys[i].chi || !sys[i].b || !sys[i].x ||
            (!sys[i].g_block && !(sys[i].k0 > 0.0 && sys[i].h > 0.0)))
            return CG_ERR_INVALID;
    std::vector<int> order(nsys);
    for (int i = 0; i < nsys; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sys[a].N > sys[b].N; });
    std::atomic<int> next(0);
    std::atomic<int> fatal(CG_OK);
    const int nw = std::min(nworkers, std::max(1, nsys));
    auto worker = [&]() {
        cg_ctx *ctx = nullptr;
        int st = cugmres_create(&ctx, device);
        if (st != CG_OK) {
            fatal = st;
            return;
        }
        if (nw > 1) cg::ctx_set_shared_gpu(ctx, true);
        for (;;) {
            const int q = next.fetch_add(1);
            if (q >= nsys) break;
            const int i = order[q];
            const cg_system &s = sys[i];
            const double t0 = now_s();
            cg_result r = {};
            st = s.g_block ? cugmres_set_operator(ctx, s.N, s.g_block, s.chi, s.chi_scale)
                           : cugmres_set_operator_green(ctx, CG_GREEN_HELMHOLTZ, s.N, s.k0, s.h, s.chi, s.chi_scale);
            if (st == CG_OK) st = cugmres_solve(ctx, s.b, s.x, opts, nullptr, 0, &r);
            r.status = st;
            r.seconds = now_s() - t0;
            results[i] = r;
            if (st == CG_ERR_CUDA || st == CG_ERR_OOM) fatal = st;
        }
        cugmres_destroy(ctx);
    };
    std::vector<std::thread> threads;
    for (int w = 0; w < nw; w++) threads.emplace_back(worker);
    for (auto &t : threads) t.join();
    return fatal.load();
}
