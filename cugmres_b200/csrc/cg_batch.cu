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
#include <math.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <map>
#include <thread>
#include <vector>

#include "../../include/cugmres.h"
#include "cg_common.cuh"
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

// ---------------------------------------------------------------------------
// Buckets: systems of one grid size solved in lockstep.
//
// cugmres_solve_buckets groups the systems by grid side N, orders each group
// by an estimate of its difficulty (optical size N k0 h sqrt(1 + max chi)
// / 2 pi, so systems of similar step counts share a bucket and few wait long
// for a slow neighbour) and cuts it into buckets of at most `max_bucket`
// systems that fit in half of the free device memory.  A bucket's arrays hold
// every system side by side (basis, intermediate T, quarter spectrum,
// contrast, x, b, and one workspace block with the DevState per system), and
// every kernel of an Arnoldi step is ONE launch for the whole bucket, the
// system being blockIdx.y (KrylovPtrs::sys_ws / sys_v, MatvecArgs::sys_*).
// A system that stops (converged, budget, breakdown) returns at once from
// every later launch of its bucket; the restart cycle (restart + 1 delayed
// CGS2 steps, back-solve, update, the next true residual and cycle decisions
// of all systems) is captured once per bucket as a CUDA graph and replayed
// with one launch per cycle, one host synchronisation per cycle.
// Scope: FP64 or mixed precision (complex64 cycles, FP64 residual and
// update), delayed CGS2, no preconditioner, A x = b (not the transposed
// system), restarted semantics; other options return CG_ERR_NOT_IMPLEMENTED.
namespace {

using namespace cg;

constexpr size_t al256(size_t v) { return (v + 255) & ~(size_t)255; }

// ||b_s|| of every system (one block per system, fixed-order reduction).
__global__ void __launch_bounds__(1024) k_bucket_nb(const double2 *__restrict__ b, long long n, char *ws,
                                                    long long sys_ws) {
    __shared__ double red[32];
    const double2 *bs = b + (long long)blockIdx.y * n;
    double acc = 0.0;
    for (long long e = threadIdx.x; e < n; e += blockDim.x) acc += bs[e].x * bs[e].x + bs[e].y * bs[e].y;
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        DevState *st = reinterpret_cast<DevState *>(ws + (long long)blockIdx.y * sys_ws);
        st->nb = sqrt(t);
    }
}

// Byte layout of one system's workspace block (every array 256-byte aligned).
struct WsLayout {
    size_t st, scale, h1, h2, Rm, cs, sn, g, y, hist, part, npart, Hm, D1, D2, tv, P, S, gpart, tickets, bytes;
};

WsLayout ws_layout(int mc, int maxit, size_t npart, size_t part, size_t gpart, size_t ngroups) {
    WsLayout w;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o = al256(o + bytes);
        return at;
    };
    w.st = take(sizeof(DevState));
    w.scale = take(sizeof(double) * (mc + 2));
    w.h1 = take(sizeof(double2) * (mc + 1));
    w.h2 = take(sizeof(double2) * (mc + 1));
    w.Rm = take(sizeof(double2) * (size_t)(mc + 1) * mc);
    w.cs = take(sizeof(double2) * mc);
    w.sn = take(sizeof(double) * mc);
    w.g = take(sizeof(double2) * (mc + 1));
    w.y = take(sizeof(double2) * mc);
    w.hist = take(sizeof(double) * ((size_t)maxit + 1));
    w.part = take(sizeof(double) * part);
    w.npart = take(sizeof(double) * npart);
    w.Hm = take(sizeof(double2) * (size_t)(mc + 1) * (mc + 1));
    w.D1 = take(sizeof(double2) * (mc + 2));
    w.D2 = take(sizeof(double2) * (mc + 2));
    w.tv = take(sizeof(double2) * (mc + 2));
    w.P = take(sizeof(double2) * (mc + 1));
    w.S = take(sizeof(double2) * (mc + 1));
    w.gpart = take(sizeof(double) * gpart);
    w.tickets = take(sizeof(unsigned int) * ngroups);
    w.bytes = o;
    return w;
}

struct BucketBufs {
    void *V = nullptr, *T = nullptr, *G = nullptr, *C = nullptr, *G32 = nullptr, *C32 = nullptr, *X = nullptr,
         *B = nullptr, *WS = nullptr;
    DevState *st_host = nullptr;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t ev = nullptr;
    ~BucketBufs() {
        if (gexec) cudaGraphExecDestroy(gexec);
        for (void *p : {V, T, G, C, G32, C32, X, B, WS})
            if (p) cudaFree(p);
        if (st_host) cudaFreeHost(st_host);
        if (cap) cudaStreamDestroy(cap);
        if (ev) cudaEventDestroy(ev);
    }
};

int cu(cudaError_t e) { return e == cudaSuccess ? CG_OK : (e == cudaErrorMemoryAllocation ? CG_ERR_OOM : CG_ERR_CUDA); }
#define BK_TRY(expr)                \
    do {                            \
        int _s = (expr);            \
        if (_s != CG_OK) return _s; \
    } while (0)
#define BK_CU(expr) BK_TRY(cu(expr))
#define BK_LAUNCH(expr)                  \
    do {                                 \
        if ((expr) != 0) return CG_ERR_CUDA; \
    } while (0)

bool host_finite(const double *p, size_t n) {
    for (size_t i = 0; i < n; i++)
        if (!std::isfinite(p[i])) return false;
    return true;
}

bool on_device(const void *p) {
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Solves the systems idx[0..B) (all of side N) as one bucket on ctx's device.
int solve_bucket(cg_ctx *ctx, const cg_system *sys, const std::vector<int> &idx, const cg_opts &o, double t_sweep,
                 cg_result *results) {
    const int nb = (int)idx.size();
    const int N = sys[idx[0]].N;
    const long long n = (long long)N * N;
    const int prec = o.precision == CG_PREC_MIXED ? 1 : 0;  // Arnoldi cycles in complex64
    const size_t esz = prec ? sizeof(float2) : sizeof(double2);
    const double t0 = now_s();
    BucketBufs bb;
    // operator of every system: the context builds it (GPU Green's block or the
    // given one, spectrum, tuned launch shapes), the bucket keeps a copy
    OpView ov{};
    size_t gq_elems = 0;
    for (int q = 0; q < nb; q++) {
        const cg_system &s = sys[idx[q]];
        const int st = s.g_block ? cugmres_set_operator(ctx, s.N, s.g_block, s.chi, s.chi_scale)
                                 : cugmres_set_operator_green(ctx, CG_GREEN_HELMHOLTZ, s.N, s.k0, s.h, s.chi,
                                                              s.chi_scale);
        if (st != CG_OK) return st;
        BK_TRY(ctx_op_view(ctx, &ov));
        if (q == 0) {
            const size_t lq = (size_t)ov.L / 2 + 1;
            gq_elems = lq * lq;
            BK_CU(cudaMalloc(&bb.G, sizeof(double2) * gq_elems * nb));
            BK_CU(cudaMalloc(&bb.C, sizeof(double) * (size_t)n * nb));
            BK_CU(cudaMalloc(&bb.X, sizeof(double2) * (size_t)n * nb));
            BK_CU(cudaMalloc(&bb.B, sizeof(double2) * (size_t)n * nb));
            if (prec) {
                BK_CU(cudaMalloc(&bb.G32, sizeof(float2) * gq_elems * nb));
                BK_CU(cudaMalloc(&bb.C32, sizeof(float) * (size_t)n * nb));
            }
        }
        if (prec) {
            BK_CU(cudaMemcpyAsync((float2 *)bb.G32 + gq_elems * q, ov.gq32, sizeof(float2) * gq_elems,
                                  cudaMemcpyDeviceToDevice, ov.stream));
            BK_CU(cudaMemcpyAsync((float *)bb.C32 + (size_t)n * q, ov.c32, sizeof(float) * n, cudaMemcpyDeviceToDevice,
                                  ov.stream));
        }
        BK_CU(cudaMemcpyAsync((double2 *)bb.G + gq_elems * q, ov.gq64, sizeof(double2) * gq_elems,
                              cudaMemcpyDeviceToDevice, ov.stream));
        BK_CU(cudaMemcpyAsync((double *)bb.C + (size_t)n * q, ov.c64, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                              ov.stream));
        if (!on_device(s.b) && !host_finite((const double *)s.b, 2 * (size_t)n)) return CG_ERR_NONFINITE;
        BK_CU(cudaMemcpyAsync((double2 *)bb.B + (size_t)n * q, s.b, sizeof(double2) * n, cudaMemcpyDefault,
                              ov.stream));
        if (o.zero_x0) {
            BK_CU(cudaMemsetAsync((double2 *)bb.X + (size_t)n * q, 0, sizeof(double2) * n, ov.stream));
        } else {
            if (!on_device(s.x) && !host_finite((const double *)s.x, 2 * (size_t)n)) return CG_ERR_NONFINITE;
            BK_CU(cudaMemcpyAsync((double2 *)bb.X + (size_t)n * q, s.x, sizeof(double2) * n, cudaMemcpyDefault,
                                  ov.stream));
        }
        // the context's buffers are rebuilt by the next set-up: wait for the copies
        BK_CU(cudaStreamSynchronize(ov.stream));
    }
    cudaStream_t s = ov.stream;
    const int L = ov.L;
    const int m = o.restart;
    const int sms_eff = std::max(1, ov.sms / nb);  // each system's share of the GPU
    const int ndot2 = dots2_blocks(prec, sms_eff, m, n);
    const int nax2 = axpy2_blocks(prec, sms_eff, m, n);
    const int nax = std::max(1, (int)std::min<long long>((n + 255) / 256, 4LL * sms_eff));
    const int rpc = rows_per_block(ov.var[0][2], L);
    const int nrb = (N + rpc - 1) / rpc;
    const size_t pld = (size_t)dots2_part_ld(m);
    const size_t ngroups = ((size_t)ndot2 + 15) / 16;
    const WsLayout wl = ws_layout(m, std::max(1, o.max_iter), std::max<size_t>(nrb, (size_t)nax) + 32,
                                  4 * (size_t)ndot2 * pld, 4 * ngroups * pld, ngroups);
    const size_t vsys = (size_t)(m + 2) * (size_t)n;
    BK_CU(cudaMalloc(&bb.V, esz * vsys * nb));
    BK_CU(cudaMalloc(&bb.T, sizeof(double2) * (size_t)N * L * nb));
    BK_CU(cudaMalloc(&bb.WS, wl.bytes * nb));
    BK_CU(cudaMemsetAsync(bb.WS, 0, wl.bytes * nb, s));
    BK_CU(cudaMallocHost((void **)&bb.st_host, sizeof(DevState) * nb));
    char *ws = (char *)bb.WS;
    KrylovPtrs kp{};
    kp.st = (DevState *)(ws + wl.st);
    kp.scale = (double *)(ws + wl.scale);
    kp.h1 = (double2 *)(ws + wl.h1);
    kp.h2 = (double2 *)(ws + wl.h2);
    kp.Rm = (double2 *)(ws + wl.Rm);
    kp.cs = (double2 *)(ws + wl.cs);
    kp.sn = (double *)(ws + wl.sn);
    kp.g = (double2 *)(ws + wl.g);
    kp.y = (double2 *)(ws + wl.y);
    kp.hist = (double *)(ws + wl.hist);
    kp.part = (double *)(ws + wl.part);
    kp.npart = (double *)(ws + wl.npart);
    kp.Hm = (double2 *)(ws + wl.Hm);
    kp.D1 = (double2 *)(ws + wl.D1);
    kp.D2 = (double2 *)(ws + wl.D2);
    kp.tv = (double2 *)(ws + wl.tv);
    kp.P = (double2 *)(ws + wl.P);
    kp.S = (double2 *)(ws + wl.S);
    kp.gpart = (double *)(ws + wl.gpart);
    kp.tickets = (unsigned int *)(ws + wl.tickets);
    kp.mcap = m;
    kp.sys_ws = (long long)wl.bytes;
    kp.sys_v = (long long)vsys;
    kp.nsys = nb;
    // initial device state of every system
    for (int q = 0; q < nb; q++) {
        DevState h;
        memset(&h, 0, sizeof(h));
        h.m = m;
        h.maxit = o.max_iter;
        h.rotation = o.givens == CG_GIVENS_REFERENCE ? 1 : 0;
        h.tol = o.tol;
        h.inner_tol = prec ? o.inner_tol : 0.0;
        h.ortho = 0;  // delayed CGS2
        BK_CU(cudaMemcpyAsync(ws + (size_t)q * wl.bytes + wl.st, &h, sizeof(h), cudaMemcpyHostToDevice, s));
        BK_CU(cudaStreamSynchronize(s));  // h lives on this stack frame
    }
    k_bucket_nb<<<dim3(1, nb), 1024, 0, s>>>((const double2 *)bb.B, n, ws + wl.st, (long long)wl.bytes);
    BK_CU(cudaGetLastError());

    // FP64 operator (true residual) and the cycles' operator (FP64, or FP32 in mixed precision)
    MatvecArgs a64;
    a64.N = N;
    a64.L = L;
    a64.vfwd = ov.var[0][0];
    a64.vcols = ov.var[0][1];
    a64.vinv = ov.var[0][2];
    a64.gq = bb.G;
    a64.cdiag = bb.C;
    a64.tw = ov.tw64;
    a64.T = bb.T;
    a64.sms = ov.sms;
    a64.nsys = nb;
    a64.sys_ws = (long long)wl.bytes;
    a64.sys_c = n;
    a64.sys_T = (long long)N * L;
    a64.sys_gq = (long long)gq_elems;
    a64.sys_b = n;
    MatvecArgs ap = a64;
    if (prec) {
        ap.vfwd = ov.var[1][0];
        ap.vcols = ov.var[1][1];
        ap.vinv = ov.var[1][2];
        ap.gq = bb.G32;
        ap.cdiag = bb.C32;
        ap.tw = ov.tw32;
    }
    VecSel vk;  // u_k of each system: V_s + k n
    vk.base = bb.V;
    vk.stride = n;
    vk.koff = 0;
    vk.sys = (long long)vsys;
    VecSel vk1 = vk;
    vk1.koff = 1;
    VecSel v0 = vk;  // V_0 of each system (the residual)
    v0.stride = 0;
    VecSel xs;
    xs.base = bb.X;
    xs.stride = 0;
    xs.koff = 0;
    xs.sys = n;

    auto enqueue_begin = [&](cudaStream_t q) -> int {
        BK_LAUNCH(launch_rows_forward(0, a64, xs, nullptr, nullptr, GATE_NONE, q));
        BK_LAUNCH(launch_cols_convolve(0, a64, nullptr, GATE_NONE, q));
        BK_LAUNCH(launch_rows_inverse(0, 1, prec, a64, xs, nullptr, bb.B, v0, kp.npart, nullptr, GATE_NONE, q));
        BK_LAUNCH(launch_cycle_begin(kp, nrb, q));
        return CG_OK;
    };
    auto enqueue_cycle = [&](cudaStream_t q) -> int {
        for (int i = 0; i < m + 1; i++) {
            BK_LAUNCH(launch_rows_forward(prec, ap, vk, nullptr, kp.st, GATE_STOP, q));
            BK_LAUNCH(launch_cols_convolve(prec, ap, kp.st, GATE_STOP, q));
            BK_LAUNCH(launch_rows_inverse(prec, 0, prec, ap, vk, nullptr, nullptr, vk1, nullptr, kp.st, GATE_STOP, q));
            BK_LAUNCH(launch_dots2(prec, bb.V, n, kp, ndot2, sms_eff, q));
            BK_LAUNCH(launch_dcgs2_step(kp, q));
            BK_LAUNCH(launch_axpy2(prec, bb.V, n, kp, nax2, sms_eff, q));
        }
        BK_LAUNCH(launch_backsolve(kp, q));
        BK_LAUNCH(launch_axpy(prec, 0, bb.V, n, kp, kp.y, 1.0, NJ_NCOL, xs, 0, 1, nax, GATE_NONE, q));
        return CG_OK;
    };
    // capture [cycle + next residual and decisions] once; replay per cycle
    BK_CU(cudaStreamCreateWithFlags(&bb.cap, cudaStreamNonBlocking));
    {
        cudaGraph_t g = nullptr;
        BK_CU(cudaStreamBeginCapture(bb.cap, cudaStreamCaptureModeThreadLocal));
        int e1 = enqueue_cycle(bb.cap);
        int e2 = e1 == CG_OK ? enqueue_begin(bb.cap) : e1;
        cudaError_t ce = cudaStreamEndCapture(bb.cap, &g);
        if (e2 != CG_OK || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return e2 != CG_OK ? e2 : CG_ERR_CUDA;
        }
        ce = cudaGraphInstantiate(&bb.gexec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            bb.gexec = nullptr;
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
    }
    BK_CU(cudaEventCreateWithFlags(&bb.ev, cudaEventDisableTiming));
    BK_TRY(enqueue_begin(s));
    std::vector<double> done_at(nb, -1.0);
    int status = CG_OK;
    // every cycle of a running system takes at least one Arnoldi step, so the
    // budget bounds the cycles; the cap only guards against a state that never
    // reports an end
    const long long max_cycles = (long long)o.max_iter + 2;
    for (long long cyc = 0;; cyc++) {
        if (cyc > max_cycles) {
            status = CG_ERR_CUDA;
            break;
        }
        BK_CU(cudaMemcpy2DAsync(bb.st_host, sizeof(DevState), ws + wl.st, wl.bytes, sizeof(DevState), nb,
                                cudaMemcpyDeviceToHost, s));
        BK_CU(cudaEventRecord(bb.ev, s));
        BK_CU(cudaEventSynchronize(bb.ev));
        const double t = now_s();
        int running = 0;
        for (int q = 0; q < nb; q++) {
            if (bb.st_host[q].status != 0) {
                if (done_at[q] < 0.0) done_at[q] = t;
            } else {
                running++;
            }
        }
        if (running == 0) break;
        if (o.timeout_s > 0.0 && t - t0 > o.timeout_s) {
            status = CG_ERR_TIMEOUT;
            break;
        }
        BK_CU(cudaGraphLaunch(bb.gexec, s));
    }
    // solutions and results
    for (int q = 0; q < nb; q++) {
        const cg_system &sy = sys[idx[q]];
        BK_CU(cudaMemcpyAsync(sy.x, (const double2 *)bb.X + (size_t)n * q, sizeof(double2) * n, cudaMemcpyDefault, s));
    }
    BK_CU(cudaStreamSynchronize(s));
    const double t1 = now_s();
    for (int q = 0; q < nb; q++) {
        const DevState &h = bb.st_host[q];
        cg_result r = {};
        switch (h.status) {
            case 1: r.status = CG_OK; break;
            case 2: r.status = CG_ERR_NOT_CONVERGED; break;
            case 3: r.status = CG_ERR_BREAKDOWN; break;
            case 4: r.status = CG_ERR_NONFINITE; break;
            default: r.status = status != CG_OK ? status : CG_ERR_CUDA; break;
        }
        r.iterations = h.it;
        r.cycles = h.cycles;
        r.rel_residual_estimate = h.est;
        r.rel_residual_true = h.true_res;
        // latency: from the bucket's start (its set-up included) to the cycle
        // boundary at which the host saw the system finish
        r.seconds = (done_at[q] > 0.0 ? done_at[q] : t1) - t0;
        results[idx[q]] = r;
    }
    (void)t_sweep;
    return CG_OK;
}

}  // namespace

extern "C" int cugmres_solve_buckets(int device, int nsys, const cg_system *sys, const cg_opts *opts_in,
                                     int max_bucket, cg_result *results) {
    if (nsys < 0 || (nsys > 0 && (!sys || !results)) || max_bucket < 0) return CG_ERR_INVALID;
    cg_opts o;
    if (opts_in) o = *opts_in;
    else cugmres_default_opts(&o);
    if (o.restart < 1 || o.max_iter < 0 || !(o.tol >= 0.0)) return CG_ERR_INVALID;
    if ((o.precision != CG_PREC_FP64 && o.precision != CG_PREC_MIXED) || o.ortho != CG_ORTHO_DCGS2 ||
        o.preconditioner != CG_PRECOND_NONE ||
        o.transpose || o.fixed_iterations || o.restart > 4500)
        return CG_ERR_NOT_IMPLEMENTED;
    for (int i = 0; i < nsys; i++)
        if (sys[i].N < 1 || !sys[i].chi || !sys[i].b || !sys[i].x ||
            (!sys[i].g_block && !(sys[i].k0 > 0.0 && sys[i].h > 0.0)))
            return CG_ERR_INVALID;
    if (nsys == 0) return CG_OK;
    const double t_sweep = now_s();
    // group by grid side, hardest first inside a group
    std::map<int, std::vector<int>, std::greater<int>> groups;
    std::vector<double> hard(nsys, 0.0);
    for (int i = 0; i < nsys; i++) {
        groups[sys[i].N].push_back(i);
        double cmax = 0.0;
        if (!on_device(sys[i].chi)) {
            const size_t nn = (size_t)sys[i].N * sys[i].N;
            for (size_t e = 0; e < nn; e++) cmax = std::max(cmax, sys[i].chi[e]);
        }
        const double kh = sys[i].k0 * sys[i].h > 0.0 ? sys[i].k0 * sys[i].h : 0.0;
        hard[i] = sys[i].N * kh * sqrt(1.0 + cmax);
    }
    cg_ctx *ctx = nullptr;
    int st = cugmres_create(&ctx, device);
    if (st != CG_OK) return st;
    cg::ctx_set_shared_gpu(ctx, true);  // lockstep launches: no persistent column pass
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = (size_t)8 << 30;
    }
    for (auto &kv : groups) {
        std::vector<int> &ids = kv.second;
        std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return hard[a] > hard[b]; });
        const int N = kv.first;
        int L = 16;
        while (L < 2 * N - 1) L *= 2;
        const long long n = (long long)N * N;
        const size_t esz = o.precision == CG_PREC_MIXED ? sizeof(float2) : sizeof(double2);
        const size_t per = esz * (size_t)(o.restart + 2) * n +
                           sizeof(double2) * ((size_t)N * L + (size_t)(L / 2 + 1) * (L / 2 + 1) + 2 * (size_t)n) +
                           sizeof(float2) * (size_t)(L / 2 + 1) * (L / 2 + 1) + (sizeof(double) + sizeof(float)) * n +
                           ((size_t)16 << 20);
        int cap = (int)std::max<size_t>(1, (free_b / 2) / per);
        if (max_bucket > 0) cap = std::min(cap, max_bucket);
        for (size_t b0 = 0; b0 < ids.size(); b0 += cap) {
            std::vector<int> bucket(ids.begin() + b0, ids.begin() + std::min(ids.size(), b0 + (size_t)cap));
            st = solve_bucket(ctx, sys, bucket, o, t_sweep, results);
            if (st != CG_OK) {
                cugmres_destroy(ctx);
                return st;
            }
        }
    }
    cugmres_destroy(ctx);
    return CG_OK;
}
