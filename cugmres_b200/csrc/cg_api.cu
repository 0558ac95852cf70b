// C-ABI of cugmres_b200: context, operator setup, matvec and the GMRES driver.
//
// The driver replaces Fast_GMRES_with_CUDA (CUDA_GMRES/GMRES.cuh:22-446).
// Differences by design:
//   * all solver state lives on the device (DevState); the host enqueues a
//     whole restart cycle and synchronises once per cycle to read the status,
//     instead of a cudaDeviceSynchronize after every kernel and two host
//     round trips per Arnoldi step (GMRES.cuh:369-371);
//   * restart, a relative tolerance and early exit are supported; the
//     reference's semantics (one cycle of exactly maxiter steps, absolute
//     tolerance gating the first step) are the fixed_iterations mode;
//   * errors are returned as status codes instead of exit() (GMRES_kernels.cuh:21-94);
//   * workspace is owned by the context and reused across solves instead of a
//     cudaMalloc/cudaFree per call (GMRES.cuh:74-76,443-444).
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include <algorithm>
#include <array>
#include <complex>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <cstddef>
#include <vector>

#include "../../include/cugmres.h"
#include "cg_common.cuh"
#include "cg_fft.cuh"
#include "cg_fno.h"
#include "cg_internal.h"

using namespace cg;

struct cg_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // operator
    bool have_op = false;
    int N = 0, L = 0;
    double2 *gq64 = nullptr;
    float2 *gq32 = nullptr;
    double *c64 = nullptr;
    float *c32 = nullptr;
    float *chi32 = nullptr;  // chi itself (without chi_scale), input of the learned preconditioner
    double2 *tw64 = nullptr;
    float2 *tw32 = nullptr;
    void *T = nullptr;  // N x L complex128 intermediate (also used as complex64)
    // Krylov workspace
    int mcap = 0;
    int itcap = 0;
    size_t vcap_bytes = 0;
    void *V = nullptr;
    DevState *st = nullptr;
    DevState *st_host = nullptr;  // pinned mirror for status reads
    KrylovPtrs kp{};
    double2 *bbuf = nullptr;  // staging of host b
    double2 *xbuf = nullptr;  // staging of host x
    double2 *rbuf = nullptr;  // FP64 vector scratch (residual, matvec staging)
    int nparts_cap = 0;
    cudaEvent_t ev = nullptr;
    // launch shapes of the three matvec passes per precision (autotuned)
    int var[2][3] = {{0, 0, 0}, {0, 0, 0}};
    // the GPU is shared with other contexts' solves (batched sweeps): the
    // autotuner leaves out the persistent column pass, which would hold every
    // SM's shared memory while the other streams' kernels wait
    bool shared_gpu = false;
    char devname[256] = {0};
    // per-phase timing
    bool prof = false;
    std::vector<cudaEvent_t> evpool;
    cg_phase_stats stats[CG_NPHASES] = {};
    // CUDA graph of one restart cycle (replayed with one launch per cycle)
    cudaStream_t cap_stream = nullptr;  // capture only; the graph is launched on `stream`
    // s-step cycles: the Hessenberg kernel of a block runs on a side stream next to
    // the next block's Newton chain (fork and join events)
    cudaStream_t side_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraphExec_t gexec = nullptr;
    unsigned char gkey[256] = {0};
    // learned preconditioner (flexible GMRES)
    cg_fno *net = nullptr;
    double k0h = 0.0;
    void *Z = nullptr;  // preconditioned basis z_j = M(v_j), restart + 1 vectors
    // s-step solves: the short delayed-CGS2 run that gives the Newton shifts
    double2 *probe_x = nullptr;  // its (discarded) iterate, N^2 values
    size_t probe_cap_bytes = 0;  // allocated bytes of probe_x (the grid side can change between solves)
    bool in_probe = false;       // that run is in progress (no graphs, no nested probe)
    size_t zcap_bytes = 0;
};

namespace cg {
void ctx_set_shared_gpu(cg_ctx *c, bool on) {
    if (c) c->shared_gpu = on;
}
int ctx_op_view(const cg_ctx *c, OpView *v) {
    if (!c || !v || !c->have_op) return CG_ERR_NO_OPERATOR;
    v->N = c->N;
    v->L = c->L;
    v->sms = c->sms;
    for (int q = 0; q < 2; q++)
        for (int p = 0; p < 3; p++) v->var[q][p] = c->var[q][p];
    v->gq64 = c->gq64;
    v->gq32 = c->gq32;
    v->c64 = c->c64;
    v->c32 = c->c32;
    v->tw64 = c->tw64;
    v->tw32 = c->tw32;
    v->stream = c->stream;
    return CG_OK;
}
}  // namespace cg

namespace {

int cuerr(cudaError_t e) { return e == cudaSuccess ? CG_OK : (e == cudaErrorMemoryAllocation ? CG_ERR_OOM : CG_ERR_CUDA); }

#define CG_TRY(expr)                  \
    do {                              \
        int _s = (expr);              \
        if (_s != CG_OK) return _s;   \
    } while (0)
#define CG_CU(expr) CG_TRY(cuerr(expr))
#define CG_LAUNCH(expr)                                  \
    do {                                                 \
        int _e = (expr);                                 \
        if (_e != 0) return CG_ERR_CUDA;                 \
    } while (0)

// CUGMRES_GRAPHS=0 launches every kernel directly instead of replaying the
// captured restart cycle.
bool graphs_enabled() {
    static const bool on = [] {
        const char *e = getenv("CUGMRES_GRAPHS");
        return !(e && e[0] == '0');
    }();
    return on;
}

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void dfree(void *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}
template <typename T> void dfree_t(T *&p) {
    void *q = (void *)p;
    dfree(q);
    p = nullptr;
}

int next_embedding(int N) {
    int L = 16;
    while (L < 2 * N - 1) L *= 2;
    return L;
}

double now_s() {
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

// ------------------------------------------------------------ setup kernels
__global__ void k_embed(const double2 *__restrict__ g, double2 *__restrict__ full, int N, int L) {
    const long long tot = (long long)L * L;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e / L), j = (int)(e % L);
        const int di = i <= L - i ? i : L - i;
        const int dj = j <= L - j ? j : L - j;
        full[e] = (di < N && dj < N) ? g[(size_t)di * N + dj] : make_double2(0.0, 0.0);
    }
}

__global__ void k_quarter(const double2 *__restrict__ full, double2 *__restrict__ q64, float2 *__restrict__ q32, int L,
                          double scale) {
    const int Lq = L / 2 + 1;
    const long long tot = (long long)Lq * Lq;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e / Lq), r = (int)(e % Lq);  // column-major quarter
        const double2 v = full[(size_t)r * L + c];
        q64[e] = make_double2(v.x * scale, v.y * scale);
        q32[e] = make_float2((float)(v.x * scale), (float)(v.y * scale));
    }
}

__global__ void k_scale_real(const double *__restrict__ a, double s, double *__restrict__ o64, float *__restrict__ o32,
                             float *__restrict__ raw32, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double v = a[e] * s;
        o64[e] = v;
        o32[e] = (float)v;
        raw32[e] = (float)a[e];
    }
}

__global__ void k_copy_c64_to_c128(const float2 *__restrict__ a, double2 *__restrict__ b, int rows, int cols, int lda) {
    const long long tot = (long long)rows * cols;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e / cols), j = (int)(e % cols);
        const float2 v = a[(size_t)i * lda + j];
        b[e] = make_double2(v.x, v.y);
    }
}

int grid_for(long long n, int cap) {
    long long g = (n + 255) / 256;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

void free_operator(cg_ctx *c) {
    dfree_t(c->gq64);
    dfree_t(c->gq32);
    dfree_t(c->c64);
    dfree_t(c->c32);
    dfree_t(c->chi32);
    dfree_t(c->tw64);
    dfree_t(c->tw32);
    dfree(c->T);
    dfree_t(c->bbuf);
    dfree_t(c->xbuf);
    dfree_t(c->rbuf);
    c->have_op = false;
}

void free_graph(cg_ctx *c) {
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
}

void free_krylov(cg_ctx *c) {
    free_graph(c);
    dfree(c->V);
    dfree_t(c->kp.scale);
    dfree_t(c->kp.h1);
    dfree_t(c->kp.h2);
    dfree_t(c->kp.Rm);
    dfree_t(c->kp.cs);
    dfree_t(c->kp.sn);
    dfree_t(c->kp.g);
    dfree_t(c->kp.y);
    dfree_t(c->kp.hist);
    dfree_t(c->kp.part);
    dfree_t(c->kp.npart);
    dfree_t(c->kp.Hm);
    dfree_t(c->kp.D1);
    dfree_t(c->kp.D2);
    dfree_t(c->kp.tv);
    dfree_t(c->kp.P);
    dfree_t(c->kp.S);
    dfree_t(c->kp.gpart);
    dfree_t(c->kp.tickets);
    dfree_t(c->kp.ss);
    dfree(c->Z);
    c->zcap_bytes = 0;
    c->mcap = 0;
    c->itcap = 0;
    c->vcap_bytes = 0;
    c->nparts_cap = 0;
}

int dot_blocks(const cg_ctx *c) { return 2 * c->sms; }
int axpy_blocks(const cg_ctx *c, long long n) { return grid_for(n, 4 * c->sms); }

// Ensures basis and small-array capacity for restart m and budget maxit.
// extra: basis slots beyond restart + 2 (an s-step block may run past the restart length)
int ensure_krylov(cg_ctx *c, int m, int maxit, size_t elem_bytes, int extra = 0) {
    const long long n = (long long)c->N * c->N;
    const size_t vbytes = (size_t)(m + 2 + extra) * (size_t)n * elem_bytes;
    const int nparts = std::max(std::max(axpy_blocks(c, n), dot_blocks(c)), std::max(c->N, 4 * c->sms));
    if (m > c->mcap || maxit > c->itcap || vbytes > c->vcap_bytes || nparts > c->nparts_cap) {
        const int mc = std::max(m, c->mcap), ic = std::max(maxit, c->itcap);
        const size_t vb = std::max(vbytes, c->vcap_bytes);
        const int np = std::max(nparts, c->nparts_cap);
        free_krylov(c);
        CG_CU(cudaMalloc(&c->V, vb));
        CG_CU(cudaMalloc((void **)&c->kp.scale, sizeof(double) * (mc + 2)));
        CG_CU(cudaMalloc((void **)&c->kp.h1, sizeof(double2) * (mc + 1)));
        CG_CU(cudaMalloc((void **)&c->kp.h2, sizeof(double2) * (mc + 1)));
        CG_CU(cudaMalloc((void **)&c->kp.Rm, sizeof(double2) * (size_t)(mc + 1) * mc));
        CG_CU(cudaMalloc((void **)&c->kp.cs, sizeof(double2) * mc));
        CG_CU(cudaMalloc((void **)&c->kp.sn, sizeof(double) * mc));
        CG_CU(cudaMalloc((void **)&c->kp.g, sizeof(double2) * (mc + 1)));
        CG_CU(cudaMalloc((void **)&c->kp.y, sizeof(double2) * mc));
        CG_CU(cudaMalloc((void **)&c->kp.hist, sizeof(double) * (ic + 1)));
        const size_t part_cgs2 = 2 * (size_t)dot_blocks(c) * (mc + 1);
        const size_t part_dcgs2 = 4 * (size_t)std::max(dots2_blocks(0, c->sms, mc, n), dots2_blocks(1, c->sms, mc, n)) *
                                  (size_t)dots2_part_ld(mc);
        const size_t nss = (size_t)sstep_part_rows(c->sms);  // most blocks of the s-step dot pass (its partial rows)
        const size_t part_ss = nss * (size_t)sstep_part_ld(mc);
        CG_CU(cudaMalloc((void **)&c->kp.part, sizeof(double) * std::max(std::max(part_cgs2, part_dcgs2), part_ss)));
        const size_t ng2 = ((size_t)std::max(dots2_blocks(0, c->sms, mc, n), dots2_blocks(1, c->sms, mc, n)) + 15) / 16;
        const size_t ngs = (nss + 15) / 16;
        const size_t ngroups = std::max(ng2, ngs);
        CG_CU(cudaMalloc((void **)&c->kp.gpart, sizeof(double) * std::max(4 * ng2 * (size_t)dots2_part_ld(mc),
                                                                          ngs * (size_t)sstep_part_ld(mc))));
        CG_CU(cudaMalloc((void **)&c->kp.tickets, sizeof(unsigned int) * ngroups));
        CG_CU(cudaMemset(c->kp.tickets, 0, sizeof(unsigned int) * ngroups));
        CG_CU(cudaMalloc((void **)&c->kp.ss, sizeof(double2) * (size_t)sstep_scratch_elems(mc)));
        CG_CU(cudaMalloc((void **)&c->kp.npart, sizeof(double) * np));
        CG_CU(cudaMalloc((void **)&c->kp.Hm, sizeof(double2) * (size_t)(mc + 1) * (mc + 1)));
        CG_CU(cudaMalloc((void **)&c->kp.D1, sizeof(double2) * (mc + 2)));
        CG_CU(cudaMalloc((void **)&c->kp.D2, sizeof(double2) * (mc + 2)));
        CG_CU(cudaMalloc((void **)&c->kp.tv, sizeof(double2) * (mc + 2)));
        CG_CU(cudaMalloc((void **)&c->kp.P, sizeof(double2) * (mc + 1)));
        CG_CU(cudaMalloc((void **)&c->kp.S, sizeof(double2) * (mc + 1)));
        c->mcap = mc;
        c->itcap = ic;
        c->vcap_bytes = vb;
        c->nparts_cap = np;
    }
    c->kp.st = c->st;
    c->kp.mcap = c->mcap;
    return CG_OK;
}

MatvecArgs margs(const cg_ctx *c, int prec, int transpose = 0) {
    MatvecArgs a;
    a.transpose = transpose;
    a.N = c->N;
    a.L = c->L;
    a.vfwd = c->var[prec][0];
    a.vcols = c->var[prec][1];
    a.vinv = c->var[prec][2];
    a.gq = prec == 0 ? (const void *)c->gq64 : (const void *)c->gq32;
    a.cdiag = prec == 0 ? (const void *)c->c64 : (const void *)c->c32;
    a.tw = prec == 0 ? (const void *)c->tw64 : (const void *)c->tw32;
    a.T = c->T;
    a.sms = c->sms;
    return a;
}

VecSel fixed_vec(const void *p) {
    VecSel v;
    v.base = const_cast<void *>(p);
    v.stride = 0;
    v.koff = 0;
    return v;
}

// blocks of the FP64 residual pass (each writes one ||r||^2 partial)
int row_blocks(const cg_ctx *c) {
    const int rpc = rows_per_block(c->var[0][2], c->L);
    return (c->N + rpc - 1) / rpc;
}

// ------------------------------------------------------------- autotuner
// Picks the launch shape of each matvec pass on the context's operator by
// coordinate descent over (forward, columns, inverse), timing whole matvecs
// with CUDA events, each after an L2 flush.  Choices are cached per process
// and in a text file (one line "device|L|precision|version fwd cols inv") under
// $CUGMRES_TUNE_CACHE, else $XDG_CACHE_HOME/cugmres_b200/autotune.txt, else
// ~/.cache/cugmres_b200/autotune.txt.  CUGMRES_AUTOTUNE=0 disables tuning;
// CUGMRES_MATVEC_SHAPE=v forces shape v.
std::mutex g_tune_mu;
std::map<std::string, std::array<int, 3>> g_tune;
bool g_tune_loaded = false;

std::string tune_path() {
    const char *e = getenv("CUGMRES_TUNE_CACHE");
    if (e && *e) return std::string(e);
    std::string base;
    const char *x = getenv("XDG_CACHE_HOME");
    if (x && *x) base = x;
    else {
        const char *h = getenv("HOME");
        base = std::string(h && *h ? h : "/tmp") + "/.cache";
    }
    return base + "/cugmres_b200/autotune.txt";
}

void tune_load() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    FILE *f = fopen(tune_path().c_str(), "r");
    if (!f) return;
    char key[512];
    int a, b, cc;
    while (fscanf(f, "%511s %d %d %d", key, &a, &b, &cc) == 4) g_tune[key] = {a, b, cc};
    fclose(f);
}

void tune_save(const std::string &key, const std::array<int, 3> &v) {
    const std::string path = tune_path();
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) {
        std::string dir = path.substr(0, slash);
        std::string cmd_dir;
        for (size_t i = 1; i <= dir.size(); i++)
            if (i == dir.size() || dir[i] == '/') {
                cmd_dir = dir.substr(0, i);
                mkdir(cmd_dir.c_str(), 0755);
            }
    }
    FILE *f = fopen(path.c_str(), "a");
    if (!f) return;
    fprintf(f, "%s %d %d %d\n", key.c_str(), v[0], v[1], v[2]);
    fclose(f);
}

int autotune(cg_ctx *c, int prec) {
    c->var[prec][0] = c->var[prec][1] = c->var[prec][2] = 0;
    const int nv = matvec_variants(c->L);
    if (nv <= 1) return CG_OK;
    const char *env = getenv("CUGMRES_AUTOTUNE");
    if (env && env[0] == '0') return CG_OK;
    // CUGMRES_MATVEC_SHAPE=v forces shape v on all three passes (diagnostics, tests)
    const char *force = getenv("CUGMRES_MATVEC_SHAPE");
    if (force && *force) {
        const int v = atoi(force);
        if (v < 0 || v >= nv) return CG_ERR_INVALID;
        for (int p = 0; p < 3; p++) c->var[prec][p] = v;
        return CG_OK;
    }
    // the key carries the tuner's version so that choices made by an older
    // tuner or for older kernels are not reused
    std::string key = std::string(c->devname) + "|" + std::to_string(c->L) + "|" + std::to_string(prec) + "|t3" +
                      (c->shared_gpu ? "s" : "");
    for (char &ch : key)
        if (ch == ' ') ch = '_';
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        tune_load();
        auto it = g_tune.find(key);
        if (it != g_tune.end() && it->second[0] < nv && it->second[1] < nv && it->second[2] < nv) {
            for (int p = 0; p < 3; p++) c->var[prec][p] = it->second[p];
            return CG_OK;
        }
    }
    const long long n = (long long)c->N * c->N;
    cudaStream_t s = c->stream;
    CG_CU(cudaMemsetAsync(c->xbuf, 0, sizeof(double2) * n, s));
    CG_CU(cudaMemsetAsync(c->T, 0, sizeof(double2) * (size_t)c->N * c->L, s));
    // In a solve the dot and axpy passes stream the Krylov basis through L2
    // between two matvecs, so each timed matvec starts after a write of twice
    // the L2 size (skipped if that buffer cannot be had).
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, c->device);
    const size_t flush_bytes = (size_t)std::max(l2, 1 << 20) * 2;
    void *flush = nullptr;
    if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
        flush = nullptr;
        cudaGetLastError();
    }
    cudaEvent_t e0, e1;
    CG_CU(cudaEventCreate(&e0));
    CG_CU(cudaEventCreate(&e1));
    int status = CG_OK;
    // time of the whole three-pass matvec (sum over timed repetitions)
    auto time_shapes = [&](const std::array<int, 3> &v) -> float {
        MatvecArgs a = margs(c, prec);
        a.vfwd = v[0];
        a.vcols = v[1];
        a.vinv = v[2];
        float tot = 0.f;
        constexpr int WARM = 2, REPS = 6;
        for (int r = 0; r < WARM + REPS && status == CG_OK; r++) {
            if (flush && cudaMemsetAsync(flush, r & 0xff, flush_bytes, s) != cudaSuccess) status = CG_ERR_CUDA;
            cudaEventRecord(e0, s);
            if (launch_rows_forward(prec, a, fixed_vec(c->xbuf), nullptr, nullptr, GATE_NONE, s) != 0 ||
                launch_cols_convolve(prec, a, nullptr, GATE_NONE, s) != 0 ||
                launch_rows_inverse(prec, 0, prec, a, fixed_vec(c->xbuf), nullptr, nullptr, fixed_vec(c->rbuf), nullptr,
                                    nullptr, GATE_NONE, s) != 0)
                status = CG_ERR_CUDA;
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) status = CG_ERR_CUDA;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (r >= WARM) tot += ms;
        }
        return tot;
    };
    // coordinate descent over the three passes, starting from shape 0
    std::array<int, 3> best = {0, 0, 0};
    float best_ms = time_shapes(best);
    for (int sweep = 0; sweep < 2 && status == CG_OK; sweep++) {
        bool changed = false;
        for (int pass = 0; pass < 3 && status == CG_OK; pass++)
            for (int v = 0; v < nv && status == CG_OK; v++) {
                if (v == best[pass] || (c->shared_gpu && matvec_variant_persistent(v))) continue;
                std::array<int, 3> cand = best;
                cand[pass] = v;
                const float ms = time_shapes(cand);
                if (ms < 0.99f * best_ms) {
                    best_ms = ms;
                    best = cand;
                    changed = true;
                }
            }
        if (!changed) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (flush) cudaFree(flush);
    if (status != CG_OK) return status;
    for (int p = 0; p < 3; p++) c->var[prec][p] = best[p];
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = best;
    tune_save(key, best);
    return CG_OK;
}

// y = A x (mode 0) or y = b - A x (mode 1) on explicit vectors, no gating.
int apply_explicit(cg_ctx *c, int prec, int mode, int out_prec, const void *x, const void *b, void *y, double *npart,
                   int transpose = 0) {
    MatvecArgs a = margs(c, prec, transpose);
    CG_LAUNCH(launch_rows_forward(prec, a, fixed_vec(x), nullptr, nullptr, GATE_NONE, c->stream));
    CG_LAUNCH(launch_cols_convolve(prec, a, nullptr, GATE_NONE, c->stream));
    CG_LAUNCH(launch_rows_inverse(prec, mode, out_prec, a, fixed_vec(x), nullptr, b, fixed_vec(y), npart, nullptr,
                                  GATE_NONE, c->stream));
    return CG_OK;
}

// Events recorded since the last collection: the interval between event i and
// event i+1 belongs to phase tag[i] of Arnoldi step iter[i] (-1: not a step).
struct CycleProf {
    std::vector<int> tag;
    std::vector<int> iter;
    int used = 0;
};

int prof_event(cg_ctx *c, int idx, cudaEvent_t *out) {
    while ((int)c->evpool.size() <= idx) {
        cudaEvent_t e;
        CG_CU(cudaEventCreate(&e));
        c->evpool.push_back(e);
    }
    *out = c->evpool[idx];
    return CG_OK;
}

// Records the event closing `phase` (the first call only opens).
int prof_mark(cg_ctx *c, CycleProf &cp, int phase, int iter, cudaStream_t s) {
    if (!c->prof) return CG_OK;
    cudaEvent_t e;
    CG_TRY(prof_event(c, cp.used, &e));
    CG_CU(cudaEventRecord(e, s));
    if (cp.used > 0) {
        cp.tag.push_back(phase);
        cp.iter.push_back(iter);
    }
    cp.used++;
    return CG_OK;
}

// Called once the stream has passed every recorded event.  steps_done: Arnoldi
// steps that did work in the cycle these events cover (later steps were gated
// off on device and move no bytes); e: element bytes of the cycle precision.
// ss > 0: the cycle ran s-step blocks of ss steps; a MATVEC interval then holds
// the block's ss matvecs and iter is the block's first basis index.
// Arnoldi steps of the run that gives an s-step solve its Newton shifts.  Measured on
// the 1024^2 GMRES(100) solve (s, S = 4 / 8): 8 steps 0.175 / 0.217, 12 steps
// 0.166 / 0.202, 16 steps 0.162 / 0.185, 24 steps 0.164 / 0.178 (shorter runs give
// rougher shifts, worse-conditioned Newton blocks and more second passes).
constexpr int SS_PROBE_STEPS = 24;

int prof_collect(cg_ctx *c, CycleProf &cp, double n, double e, int steps_done, bool delayed, int ss = 0,
                 bool chained = false) {
    if (c->prof && cp.used >= 2) {
        // s-step: a block that skipped its second Gram-Schmidt pass moved no bytes in
        // its second dot and update launches (the second of each per block start k)
        std::vector<int> skipped;
        std::map<int, int> seen_dots, seen_axpy;
        if (ss > 0) CG_TRY(sstep_skipped(c->kp, c->mcap / ss + 1, skipped, c->stream));
        for (int i = 0; i + 1 < cp.used; i++) {
            float ms = 0.f;
            CG_CU(cudaEventElapsedTime(&ms, c->evpool[i], c->evpool[i + 1]));
            const int t = cp.tag[i], k = cp.iter[i];
            bool live = k < steps_done;
            if (ss > 0 && k >= 0 && (t == CG_PHASE_DOTS || t == CG_PHASE_AXPY)) {
                const int nth = (t == CG_PHASE_DOTS ? seen_dots : seen_axpy)[k]++;
                const int blk = k / ss;
                if (nth == 1 && blk < (int)skipped.size() && skipped[blk]) live = false;
            }
            double bytes = 0.0;
            switch (ss > 0 ? -t - 100 : t) {
                case CG_PHASE_MATVEC: bytes = live ? 16.0 * n * e : 0.0; break;
                case CG_PHASE_DOTS: bytes = live ? (k + 2.0) * n * e : 0.0; break;
                case CG_PHASE_AXPY: bytes = live ? (k + (delayed ? 4.0 : 3.0)) * n * e : 0.0; break;
                case -CG_PHASE_MATVEC - 100:
                    // a fused chain does not read w_1 .. w_{S-1} back: one vector less per chained matvec
                    bytes = live ? (16.0 * ss - (chained ? ss - 1.0 : 0.0)) * n * e : 0.0;
                    break;
                case -CG_PHASE_DOTS - 100: bytes = live ? (k + 1.0 + ss) * n * e : 0.0; break;  // Q^H W and W^H W
                case -CG_PHASE_AXPY - 100: bytes = live ? (k + 1.0 + 2.0 * ss) * n * e : 0.0; break;  // W <- W A - Q B
                case -CG_PHASE_UPDATE - 100: bytes = steps_done * n * e + 2.0 * n * 16.0; break;
                case -CG_PHASE_RESIDUAL - 100: bytes = 16.0 * n * 16.0; break;
                case CG_PHASE_UPDATE: bytes = (steps_done - (delayed ? 1 : 0)) * n * e + 2.0 * n * 16.0; break;
                case CG_PHASE_RESIDUAL: bytes = 16.0 * n * 16.0; break;
                default: bytes = 0.0;
            }
            if (t >= 0 && t < CG_NPHASES) {
                c->stats[t].ms += ms;
                c->stats[t].bytes += bytes;
                c->stats[t].launches += (t == CG_PHASE_SMALL || live || t == CG_PHASE_UPDATE || t == CG_PHASE_RESIDUAL) ? 1 : 0;
            }
        }
    }
    cp.used = 0;
    cp.tag.clear();
    cp.iter.clear();
    return CG_OK;
}

// Eigenvalues of the leading n x n block of a complex upper Hessenberg matrix
// (row-major, leading dimension ld): shifted QR iteration with Wilkinson
// shifts, unitary Givens rotations and deflation at negligible subdiagonal
// entries (Golub and Van Loan, Matrix Computations, 4th ed., sec. 7.5).  Only
// the active window is updated, since only eigenvalues are wanted.
std::vector<std::complex<double>> hessenberg_eigenvalues(const std::vector<double2> &Hin, int n, int ld) {
    typedef std::complex<double> cd;
    std::vector<cd> H((size_t)n * n, cd(0.0, 0.0)), ev(n);
    for (int i = 0; i < n; i++)
        for (int j = std::max(0, i - 1); j < n; j++) H[(size_t)i * n + j] = cd(Hin[(size_t)i * ld + j].x, Hin[(size_t)i * ld + j].y);
    auto at = [&](int i, int j) -> cd & { return H[(size_t)i * n + j]; };
    int hi = n - 1, iter = 0;
    std::vector<cd> cs(n), sn(n);
    while (hi >= 0) {
        if (hi == 0) {
            ev[0] = at(0, 0);
            break;
        }
        int lo = hi;
        while (lo > 0) {
            const double sc = std::abs(at(lo - 1, lo - 1)) + std::abs(at(lo, lo));
            if (std::abs(at(lo, lo - 1)) <= 1e-14 * (sc > 0.0 ? sc : 1.0)) break;
            lo--;
        }
        if (lo == hi) {
            ev[hi] = at(hi, hi);
            hi--;
            iter = 0;
            continue;
        }
        if (++iter > 100) {  // no convergence: the diagonal of the window stands in
            for (int i = lo; i <= hi; i++) ev[i] = at(i, i);
            hi = lo - 1;
            iter = 0;
            continue;
        }
        const cd a = at(hi - 1, hi - 1), b = at(hi - 1, hi), c = at(hi, hi - 1), d = at(hi, hi);
        const cd tr = a + d, det = a * d - b * c, disc = std::sqrt(tr * tr * 0.25 - det);
        const cd m1 = tr * 0.5 + disc, m2 = tr * 0.5 - disc;
        cd mu = std::abs(m1 - d) < std::abs(m2 - d) ? m1 : m2;
        if (iter % 11 == 10) mu = d + 0.75 * std::abs(c);  // exceptional shift
        for (int i = lo; i <= hi; i++) at(i, i) -= mu;
        for (int j = lo; j < hi; j++) {
            const cd x = at(j, j), y = at(j + 1, j);
            const double r = std::sqrt(std::norm(x) + std::norm(y));
            const cd cc = r > 0.0 ? x / r : cd(1.0, 0.0), ss = r > 0.0 ? y / r : cd(0.0, 0.0);
            for (int k2 = j; k2 <= hi; k2++) {
                const cd u = at(j, k2), v = at(j + 1, k2);
                at(j, k2) = std::conj(cc) * u + std::conj(ss) * v;
                at(j + 1, k2) = -ss * u + cc * v;
            }
            cs[j] = cc;
            sn[j] = ss;
        }
        for (int j = lo; j < hi; j++) {
            const cd cc = cs[j], ss = sn[j];
            for (int i = lo; i <= std::min(j + 2, hi); i++) {
                const cd u = at(i, j), v = at(i, j + 1);
                at(i, j) = u * cc + v * ss;
                at(i, j + 1) = -u * std::conj(ss) + v * std::conj(cc);
            }
        }
        for (int i = lo; i <= hi; i++) at(i, i) += mu;
    }
    return ev;
}

// The first `count` points of a (modified) Leja ordering of `pts`: the largest
// in modulus, then each next one maximising the product of distances to those
// already taken (as logarithms); well-spread shifts keep the Newton basis of
// the s-step blocks well conditioned (Reichel, BIT 30 (1990)).
std::vector<std::complex<double>> leja_points(std::vector<std::complex<double>> pts, int count) {
    std::vector<std::complex<double>> out;
    if (pts.empty()) return out;
    size_t first = 0;
    for (size_t i = 1; i < pts.size(); i++)
        if (std::abs(pts[i]) > std::abs(pts[first])) first = i;
    out.push_back(pts[first]);
    pts.erase(pts.begin() + first);
    while ((int)out.size() < count && !pts.empty()) {
        size_t best = 0;
        double bv = -1e300;
        for (size_t i = 0; i < pts.size(); i++) {
            double v = 0.0;
            for (const auto &q : out) v += std::log(std::abs(pts[i] - q) + 1e-300);
            if (v > bv) {
                bv = v;
                best = i;
            }
        }
        out.push_back(pts[best]);
        pts.erase(pts.begin() + best);
    }
    while ((int)out.size() < count) out.push_back(out.back());
    return out;
}

bool all_finite(const double *p, size_t n) {
    for (size_t i = 0; i < n; i++)
        if (!isfinite(p[i])) return false;
    return true;
}

}  // namespace

// ================================================================== C-ABI
extern "C" {

const char *cugmres_strerror(int s) {
    switch (s) {
        case CG_OK: return "ok";
        case CG_ERR_INVALID: return "invalid argument";
        case CG_ERR_CUDA: return "CUDA runtime error";
        case CG_ERR_NOT_CONVERGED: return "not converged within the iteration budget";
        case CG_ERR_BREAKDOWN: return "Arnoldi breakdown without convergence";
        case CG_ERR_NONFINITE: return "non-finite value in input or iteration";
        case CG_ERR_TIMEOUT: return "timeout";
        case CG_ERR_NOT_IMPLEMENTED: return "not implemented for these sizes/options";
        case CG_ERR_NO_OPERATOR: return "operator not set";
        case CG_ERR_OOM: return "device out of memory";
        default: return "unknown status";
    }
}

int cugmres_version(void) { return 100; }

void cugmres_default_opts(cg_opts *o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->restart = 100;
    o->max_iter = 10000;
    o->tol = 1e-10;
    o->precision = CG_PREC_FP64;
    o->givens = CG_GIVENS_UNITARY;
    o->inner_tol = 1e-5;
    o->zero_x0 = 0;
    o->fixed_iterations = 0;
    o->timeout_s = 0.0;
    o->ortho = CG_ORTHO_DCGS2;
}

int cugmres_create(cg_ctx **out, int device) {
    if (!out) return CG_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    CG_CU(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return CG_ERR_INVALID;
    CG_CU(cudaSetDevice(device));
    cg_ctx *c = new cg_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
            strncpy(c->devname, prop.name, sizeof(c->devname) - 1);
        }
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return CG_ERR_CUDA;
    }
    c->own_stream = true;
    if (cudaMalloc((void **)&c->st, sizeof(DevState)) != cudaSuccess ||
        cudaMallocHost((void **)&c->st_host, sizeof(DevState)) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev, cudaEventDisableTiming) != cudaSuccess) {
        cugmres_destroy(c);
        return CG_ERR_CUDA;
    }
    cudaMemset(c->st, 0, sizeof(DevState));
    *out = c;
    return CG_OK;
}

int cugmres_destroy(cg_ctx *c) {
    if (!c) return CG_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_operator(c);
    free_krylov(c);
    dfree_t(c->st);
    if (c->st_host) cudaFreeHost(c->st_host);
    if (c->ev) cudaEventDestroy(c->ev);
    for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
    free_graph(c);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    if (c->side_stream) cudaStreamDestroy(c->side_stream);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    dfree_t(c->probe_x);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return CG_OK;
}

int cugmres_set_stream(cg_ctx *c, void *stream) {
    if (!c) return CG_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->own_stream && c->stream) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return CG_OK;
}

int cugmres_synchronize(cg_ctx *c) {
    if (!c) return CG_ERR_INVALID;
    return cuerr(cudaStreamSynchronize(c->stream));
}

int cugmres_profile(cg_ctx *c, int enable) {
    if (!c) return CG_ERR_INVALID;
    c->prof = enable != 0;
    for (int i = 0; i < CG_NPHASES; i++) c->stats[i] = cg_phase_stats{0.0, 0.0, 0};
    return CG_OK;
}

int cugmres_profile_read(cg_ctx *c, cg_phase_stats *out) {
    if (!c || !out) return CG_ERR_INVALID;
    for (int i = 0; i < CG_NPHASES; i++) out[i] = c->stats[i];
    return CG_OK;
}

int cugmres_matvec_shapes(const cg_ctx *c, int precision, int *shapes) {
    if (!c || !shapes || (precision != CG_PREC_FP64 && precision != CG_PREC_MIXED)) return CG_ERR_INVALID;
    if (!c->have_op) return CG_ERR_NO_OPERATOR;
    const int p = precision == CG_PREC_FP64 ? 0 : 1;
    for (int i = 0; i < 3; i++) shapes[i] = c->var[p][i];
    return CG_OK;
}

int cugmres_set_preconditioner(cg_ctx *c, cg_fno *net, double k0h) {
    if (!c || (net && !(k0h > 0.0 && isfinite(k0h)))) return CG_ERR_INVALID;
    if (net && fno::device_of(net) != c->device) return CG_ERR_INVALID;
    c->net = net;
    c->k0h = net ? k0h : 0.0;
    return CG_OK;
}

int cugmres_grid_size(const cg_ctx *c, int *N, int *L) {
    if (!c || !c->have_op) return CG_ERR_NO_OPERATOR;
    if (N) *N = c->N;
    if (L) *L = c->L;
    return CG_OK;
}

static int set_operator_dev(cg_ctx *c, int N, const double2 *g_dev, const double *chi_dev, double chi_scale) {
    const int L = c->L;
    const long long n = (long long)N * N;
    // spectrum: even embedding, full FP64 2D transform, quarter with 1/L^2 folded in
    double2 *full = nullptr;
    CG_CU(cudaMalloc((void **)&full, sizeof(double2) * (size_t)L * L));
    k_embed<<<grid_for((long long)L * L, 8 * c->sms), 256, 0, c->stream>>>(g_dev, full, N, L);
    int e = launch_fft2d_full_fp64(L, full, c->tw64, c->stream);
    if (e == 0) {
        k_quarter<<<grid_for((long long)(L / 2 + 1) * (L / 2 + 1), 8 * c->sms), 256, 0, c->stream>>>(
            full, c->gq64, c->gq32, L, 1.0 / ((double)L * (double)L));
        k_scale_real<<<grid_for(n, 8 * c->sms), 256, 0, c->stream>>>(chi_dev, chi_scale, c->c64, c->c32, c->chi32, n);
    }
    cudaError_t ce = cudaStreamSynchronize(c->stream);
    cudaFree(full);
    if (e != 0) return CG_ERR_CUDA;
    return cuerr(ce);
}

int cugmres_set_operator(cg_ctx *c, int N, const cg_c128 *g_block, const double *chi, double chi_scale) {
    if (!c || !g_block || !chi || N < 1 || !isfinite(chi_scale)) return CG_ERR_INVALID;
    const int L = next_embedding(N);
    if (!fft_supported(L)) return CG_ERR_NOT_IMPLEMENTED;
    CG_CU(cudaSetDevice(c->device));
    const long long n = (long long)N * N;
    const bool g_dev = is_device_ptr(g_block), chi_dev = is_device_ptr(chi);
    if (!g_dev && !all_finite((const double *)g_block, 2 * (size_t)n)) return CG_ERR_NONFINITE;
    if (!chi_dev && !all_finite(chi, (size_t)n)) return CG_ERR_NONFINITE;
    // a context keeps its buffers when the grid size does not change (batched sweeps)
    const bool same = c->gq64 != nullptr && c->N == N && c->L == L;
    c->have_op = false;
    if (!same) {
        free_operator(c);
        free_krylov(c);
        c->N = N;
        c->L = L;
        const int Lq = L / 2 + 1;
        CG_CU(cudaMalloc((void **)&c->gq64, sizeof(double2) * (size_t)Lq * Lq));
        CG_CU(cudaMalloc((void **)&c->gq32, sizeof(float2) * (size_t)Lq * Lq));
        CG_CU(cudaMalloc((void **)&c->c64, sizeof(double) * n));
        CG_CU(cudaMalloc((void **)&c->c32, sizeof(float) * n));
        CG_CU(cudaMalloc((void **)&c->chi32, sizeof(float) * n));
        CG_CU(cudaMalloc((void **)&c->tw64, sizeof(double2) * 4 * L));
        CG_CU(cudaMalloc((void **)&c->tw32, sizeof(float2) * 4 * L));
        CG_CU(cudaMalloc(&c->T, sizeof(double2) * (size_t)N * L));
        CG_CU(cudaMalloc((void **)&c->bbuf, sizeof(double2) * n));
        CG_CU(cudaMalloc((void **)&c->xbuf, sizeof(double2) * n));
        CG_CU(cudaMalloc((void **)&c->rbuf, sizeof(double2) * n));
    }
    // per-stage twiddle tables (cg_fft.cuh layout) of the 16- and 8-point
    // plans, forward exp(-2 pi i m / L) and inverse, computed in double
    std::vector<double2> tw(4 * L);
    std::vector<float2> twf(4 * L);
    const double pi = 3.14159265358979323846;
    for (int t = 0; t < 4; t++) {
        const double sg = (t & 1) ? 1.0 : -1.0;
        for (int i = 0; i < L; i++) {
            const int m = twiddle_exponent(L, t < 2 ? 16 : 8, i);
            const double a = 2.0 * pi * (double)(m < 0 ? 0 : m) / (double)L;
            tw[(size_t)t * L + i] = m < 0 ? make_double2(0.0, 0.0) : make_double2(cos(a), sg * sin(a));
        }
    }
    for (size_t i = 0; i < tw.size(); i++) twf[i] = make_float2((float)tw[i].x, (float)tw[i].y);
    CG_CU(cudaMemcpyAsync(c->tw64, tw.data(), sizeof(double2) * 4 * L, cudaMemcpyHostToDevice, c->stream));
    CG_CU(cudaMemcpyAsync(c->tw32, twf.data(), sizeof(float2) * 4 * L, cudaMemcpyHostToDevice, c->stream));
    double2 *g_tmp = nullptr;
    double *chi_tmp = nullptr;
    const double2 *gp = (const double2 *)g_block;
    const double *cp = chi;
    if (!g_dev) {
        CG_CU(cudaMalloc((void **)&g_tmp, sizeof(double2) * n));
        CG_CU(cudaMemcpyAsync(g_tmp, g_block, sizeof(double2) * n, cudaMemcpyHostToDevice, c->stream));
        gp = g_tmp;
    }
    if (!chi_dev) {
        CG_CU(cudaMalloc((void **)&chi_tmp, sizeof(double) * n));
        CG_CU(cudaMemcpyAsync(chi_tmp, chi, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
        cp = chi_tmp;
    }
    int s = set_operator_dev(c, N, gp, cp, chi_scale);
    if (g_tmp) cudaFree(g_tmp);
    if (chi_tmp) cudaFree(chi_tmp);
    if (s != CG_OK) return s;
    CG_TRY(autotune(c, 0));
    CG_TRY(autotune(c, 1));
    c->have_op = true;
    return CG_OK;
}

static int green_args_ok(int kind, int N, double k0, double h) {
    if (N < 1) return 0;
    if (kind == CG_GREEN_REFERENCE) return 1;
    if (kind == CG_GREEN_PYGMRES) return k0 > 0.0 && isfinite(k0);
    if (kind == CG_GREEN_HELMHOLTZ) return k0 > 0.0 && h > 0.0 && isfinite(k0) && isfinite(h);
    return 0;
}

int cugmres_green_block_device(int kind, int N, double k0, double h, cg_c128 *out, void *stream) {
    if (!out || !green_args_ok(kind, N, k0, h)) return CG_ERR_INVALID;
    if (!is_device_ptr(out)) return CG_ERR_INVALID;
    int dev = 0, sms = 148;
    CG_CU(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    CG_LAUNCH(launch_green_block(kind, N, k0, h, (double2 *)out, sms, (cudaStream_t)stream));
    return CG_OK;
}

int cugmres_set_operator_green(cg_ctx *c, int kind, int N, double k0, double h, const double *chi, double chi_scale) {
    if (!c || !chi || !green_args_ok(kind, N, k0, h) || !isfinite(chi_scale)) return CG_ERR_INVALID;
    CG_CU(cudaSetDevice(c->device));
    double2 *g = nullptr;
    CG_CU(cudaMalloc((void **)&g, sizeof(double2) * (size_t)N * N));
    int st = launch_green_block(kind, N, k0, h, g, c->sms, c->stream) ? CG_ERR_CUDA : CG_OK;
    if (st == CG_OK) st = cugmres_set_operator(c, N, (const cg_c128 *)g, chi, chi_scale);
    cudaStreamSynchronize(c->stream);
    cudaFree(g);
    return st;
}

int cugmres_set_operator_circulant(cg_ctx *c, int N, const cg_c64 *g_prep, const double *chi, double chi_scale) {
    if (!c || !g_prep || N < 1) return CG_ERR_INVALID;
    const int M = 2 * N - 1;
    std::vector<cg_c128> g((size_t)N * N);
    if (is_device_ptr(g_prep)) {
        std::vector<cg_c64> tmp((size_t)M * M);
        CG_CU(cudaMemcpy(tmp.data(), g_prep, sizeof(cg_c64) * tmp.size(), cudaMemcpyDeviceToHost));
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) g[(size_t)i * N + j] = {tmp[(size_t)i * M + j].re, tmp[(size_t)i * M + j].im};
    } else {
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++)
                g[(size_t)i * N + j] = {g_prep[(size_t)i * M + j].re, g_prep[(size_t)i * M + j].im};
    }
    return cugmres_set_operator(c, N, g.data(), chi, chi_scale);
}

static int matvec_impl(cg_ctx *c, const void *x, void *y, int precision, int transpose) {
    if (!c || !x || !y) return CG_ERR_INVALID;
    if (!c->have_op) return CG_ERR_NO_OPERATOR;
    if (precision != CG_PREC_FP64 && precision != CG_PREC_MIXED) return CG_ERR_INVALID;
    CG_CU(cudaSetDevice(c->device));
    const int prec = precision == CG_PREC_FP64 ? 0 : 1;
    const size_t es = prec == 0 ? sizeof(double2) : sizeof(float2);
    const size_t bytes = es * (size_t)c->N * c->N;
    const bool xd = is_device_ptr(x), yd = is_device_ptr(y);
    const void *xp = x;
    void *yp = y;
    if (!xd) {
        CG_CU(cudaMemcpyAsync(c->xbuf, x, bytes, cudaMemcpyHostToDevice, c->stream));
        xp = c->xbuf;
    }
    if (!yd) yp = c->rbuf;
    CG_TRY(apply_explicit(c, prec, 0, prec, xp, nullptr, yp, nullptr, transpose));
    if (!yd) CG_CU(cudaMemcpyAsync(y, yp, bytes, cudaMemcpyDeviceToHost, c->stream));
    return cuerr(cudaStreamSynchronize(c->stream));
}

int cugmres_matvec(cg_ctx *c, const void *x, void *y, int precision) { return matvec_impl(c, x, y, precision, 0); }

int cugmres_matvec_transpose(cg_ctx *c, const void *x, void *y, int precision) {
    return matvec_impl(c, x, y, precision, 1);
}

int cugmres_residual(cg_ctx *c, const cg_c128 *b, const cg_c128 *x, cg_c128 *r, double *rel) {
    if (!c || !b || !x) return CG_ERR_INVALID;
    if (!c->have_op) return CG_ERR_NO_OPERATOR;
    CG_CU(cudaSetDevice(c->device));
    const long long n = (long long)c->N * c->N;
    const size_t bytes = sizeof(double2) * n;
    CG_TRY(ensure_krylov(c, 1, 1, sizeof(double2)));
    const void *bp = b, *xp = x;
    if (!is_device_ptr(b)) {
        CG_CU(cudaMemcpyAsync(c->bbuf, b, bytes, cudaMemcpyHostToDevice, c->stream));
        bp = c->bbuf;
    }
    if (!is_device_ptr(x)) {
        CG_CU(cudaMemcpyAsync(c->xbuf, x, bytes, cudaMemcpyHostToDevice, c->stream));
        xp = c->xbuf;
    }
    void *rp = (r && is_device_ptr(r)) ? (void *)r : (void *)c->rbuf;
    CG_TRY(apply_explicit(c, 0, 1, 0, xp, bp, rp, c->kp.npart));
    const int nb = row_blocks(c);
    std::vector<double> parts(nb);
    CG_CU(cudaMemcpyAsync(parts.data(), c->kp.npart, sizeof(double) * nb, cudaMemcpyDeviceToHost, c->stream));
    if (r && rp == c->rbuf) CG_CU(cudaMemcpyAsync(r, rp, bytes, cudaMemcpyDeviceToHost, c->stream));
    CG_TRY(launch_norm2(0, bp, n, c->kp.npart, &c->st->counter[2], &c->st->scalar, axpy_blocks(c, n), c->stream) ? CG_ERR_CUDA : CG_OK);
    double nb2 = 0.0;
    CG_CU(cudaMemcpyAsync(&nb2, &c->st->scalar, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CG_CU(cudaStreamSynchronize(c->stream));
    double rr = 0.0;
    for (int i = 0; i < nb; i++) rr += parts[i];
    if (rel) *rel = sqrt(rr) / nb2;
    return CG_OK;
}

int cugmres_solve(cg_ctx *c, const cg_c128 *b, cg_c128 *x, const cg_opts *opts_in, double *res_hist, int res_hist_len,
                  cg_result *result) {
    const double t0 = now_s();
    if (!c || !b || !x) return CG_ERR_INVALID;
    if (!c->have_op) return CG_ERR_NO_OPERATOR;
    cg_opts o;
    if (opts_in) o = *opts_in;
    else cugmres_default_opts(&o);
    if (o.restart < 1 || o.max_iter < 0 || !(o.tol >= 0.0) || (o.precision != CG_PREC_FP64 && o.precision != CG_PREC_MIXED) ||
        (o.givens != CG_GIVENS_UNITARY && o.givens != CG_GIVENS_REFERENCE) ||
        (o.ortho != CG_ORTHO_DCGS2 && o.ortho != CG_ORTHO_CGS2 && o.ortho != CG_ORTHO_SSTEP) ||
        (o.preconditioner != CG_PRECOND_NONE && o.preconditioner != CG_PRECOND_LEARNED))
        return CG_ERR_INVALID;
    const bool learned = o.preconditioner == CG_PRECOND_LEARNED;
    // s-step Arnoldi: S steps per block; the shifts are Ritz values of a short delayed-CGS2 run
    const bool sstep = o.ortho == CG_ORTHO_SSTEP;
    const int S = sstep ? (o.sstep > 0 ? o.sstep : 4) : 0;
    if (sstep && (!sstep_supported(S) || learned || o.fixed_iterations || o.givens != CG_GIVENS_UNITARY ||
                  o.restart < S))
        return CG_ERR_INVALID;
    if (learned && !c->net) return CG_ERR_INVALID;
    if (learned && o.transpose) return CG_ERR_NOT_IMPLEMENTED;  // the network approximates A^-1, not A^-T
    if (learned && (c->N < 32 || c->N > 1024)) return CG_ERR_NOT_IMPLEMENTED;
    // per-cycle coefficient arrays live in shared memory (<= 227 KB per block)
    if (o.restart > 4500 || (o.fixed_iterations && o.max_iter > 4500)) return CG_ERR_NOT_IMPLEMENTED;
    CG_CU(cudaSetDevice(c->device));
    const int prec = o.precision == CG_PREC_FP64 ? 0 : 1;
    const int m = o.fixed_iterations ? std::max(1, o.max_iter) : o.restart;
    const long long n = (long long)c->N * c->N;
    const size_t bytes = sizeof(double2) * n;
    const size_t esz = prec == 0 ? sizeof(double2) : sizeof(float2);
    CG_TRY(ensure_krylov(c, m, std::max(1, o.max_iter), esz, S));
    cudaStream_t s = c->stream;
    if (learned) {
        // flexible GMRES keeps z_j = M(v_j) next to the basis
        const size_t zb = (size_t)(m + 1) * (size_t)n * esz;
        if (c->zcap_bytes < zb) {
            dfree(c->Z);
            c->zcap_bytes = 0;
            CG_CU(cudaMalloc(&c->Z, zb));
            c->zcap_bytes = zb;
        }
        CG_TRY(fno::prepare(c->net, c->N, (float)c->k0h));
    }

    // inputs
    const bool bd = is_device_ptr(b), xd = is_device_ptr(x);
    if (!bd && !all_finite((const double *)b, 2 * (size_t)n)) return CG_ERR_NONFINITE;
    if (!xd && !o.zero_x0 && !all_finite((const double *)x, 2 * (size_t)n)) return CG_ERR_NONFINITE;
    const double2 *bp = (const double2 *)b;
    double2 *xp = (double2 *)x;
    if (!bd) {
        CG_CU(cudaMemcpyAsync(c->bbuf, b, bytes, cudaMemcpyHostToDevice, s));
        bp = c->bbuf;
    }
    if (!xd) {
        xp = c->xbuf;
        if (!o.zero_x0) CG_CU(cudaMemcpyAsync(xp, x, bytes, cudaMemcpyHostToDevice, s));
    }
    if (o.zero_x0) CG_CU(cudaMemsetAsync(xp, 0, bytes, s));

    // s-step: the Newton shifts are the Leja-ordered Ritz values of a short
    // delayed-CGS2 run from b (the outer Ritz values, which Arnoldi finds first),
    // made before the solve and not counted in it, so every restart cycle of the
    // solve runs s-step blocks; without enough columns the first cycle of the
    // solve runs delayed CGS2 and gives them instead
    double2 shifts_probe[SS_MAX];
    bool probe_ok = false;
    if (sstep && !c->in_probe) {
        const int p = std::min(m, SS_PROBE_STEPS);
        if (c->probe_cap_bytes < bytes) {
            dfree_t(c->probe_x);
            c->probe_cap_bytes = 0;
            CG_CU(cudaMalloc((void **)&c->probe_x, bytes));
            c->probe_cap_bytes = bytes;
        }
        cg_opts po = o;
        po.ortho = CG_ORTHO_DCGS2;
        po.precision = CG_PREC_FP64;
        po.restart = p;
        po.max_iter = p;
        po.tol = 0.0;
        po.zero_x0 = 1;
        po.fixed_iterations = 0;
        po.preconditioner = CG_PRECOND_NONE;
        po.timeout_s = 0.0;
        cg_result pres;
        c->in_probe = true;
        const int pe = cugmres_solve(c, (const cg_c128 *)bp, (cg_c128 *)c->probe_x, &po, nullptr, 0, &pres);
        c->in_probe = false;
        if (pe != CG_OK && pe != CG_ERR_NOT_CONVERGED) return pe;
        const int ncol = std::min(pres.iterations, p);
        if (ncol >= S) {
            const int ld = c->mcap + 1;
            std::vector<double2> hm((size_t)ncol * ld);
            CG_CU(cudaMemcpyAsync(hm.data(), c->kp.Hm, sizeof(double2) * hm.size(), cudaMemcpyDeviceToHost, s));
            CG_CU(cudaStreamSynchronize(s));
            const std::vector<std::complex<double>> ritz = hessenberg_eigenvalues(hm, ncol, ld);
            bool fin = true;
            for (const auto &z : ritz) fin = fin && std::isfinite(z.real()) && std::isfinite(z.imag());
            if (fin) {
                const std::vector<std::complex<double>> th = leja_points(ritz, S);
                for (int i = 0; i < SS_MAX; i++)
                    shifts_probe[i] = i < S ? make_double2(th[i].real(), th[i].imag()) : make_double2(0.0, 0.0);
                probe_ok = true;
            }
        }
    }

    // device state
    DevState h;
    memset(&h, 0, sizeof(h));
    h.m = m;
    h.maxit = o.max_iter;
    h.rotation = o.givens == CG_GIVENS_REFERENCE ? 1 : 0;
    h.fixed = o.fixed_iterations ? 1 : 0;
    h.tol = o.tol;
    h.inner_tol = prec == 1 ? o.inner_tol : 0.0;
    // the flexible variant stores z_j explicitly, so it uses the CGS2 path (the delayed
    // reorthogonalisation would need A M(.) to be linear)
    // (flexible GMRES: preconditioned cycles CGS2, plain cycles the requested scheme)
    h.ortho = (o.ortho == CG_ORTHO_CGS2 || learned) ? 1 : 0;
    const bool want_delayed = o.ortho == CG_ORTHO_DCGS2;
    bool delayed = h.ortho == 0;  // scheme of the cycle being enqueued
    *c->st_host = h;
    CG_CU(cudaMemcpyAsync(c->st, c->st_host, sizeof(DevState), cudaMemcpyHostToDevice, s));
    CG_LAUNCH(launch_norm2(0, bp, n, c->kp.npart, &c->st->counter[2], &c->st->nb, axpy_blocks(c, n), s));

    KrylovPtrs kp = c->kp;
    MatvecArgs a64 = margs(c, 0, o.transpose ? 1 : 0);
    MatvecArgs ap = margs(c, prec, o.transpose ? 1 : 0);
    VecSel vk;  // V_k (input of the Arnoldi matvec)
    vk.base = c->V;
    vk.stride = n;
    vk.koff = 0;
    VecSel vk1 = vk;  // V_{k+1}
    vk1.koff = 1;
    VecSel xs = fixed_vec(xp);
    VecSel zk = vk;  // Z_k (input of the flexible Arnoldi matvec)
    zk.base = c->Z;
    const int nrb = row_blocks(c);
    const int ndot = dot_blocks(c), nax = axpy_blocks(c, n), ndot2 = dots2_blocks(prec, c->sms, c->mcap, n);
    const int nax2 = axpy2_blocks(prec, c->sms, c->mcap, n);
    int status = CG_OK;

    int prec_cycles = 0, x0_learned = 0;
    // Preconditioner policy: the first cycle runs preconditioned, the second plain;
    // afterwards each cycle uses the mode whose last cycle cut the true residual
    // faster per second (log reduction / wall time); a preconditioned cycle that
    // does not reduce it at all switches to plain GMRES for the rest of the solve.
    // Preconditioned cycles, and the plain probe, last at most LEARNED_CYCLE_STEPS
    // steps: each preconditioned cycle refreshes the measured rate, so a choice
    // that the first (easiest) cycle biased towards the network costs at most
    // that many expensive steps, and a long restart or an unrestarted solve does
    // not spend its budget on the network before the modes are compared.
    constexpr int LEARNED_CYCLE_STEPS = 40;
    double rate_prec = -1.0, rate_plain = -1.0;  // < 0: not measured yet
    bool cycle_open = false, last_prec = false, prec_failed = false;
    double cycle_t0 = 0.0, cycle_res0 = 0.0;
    if (learned && o.learned_x0 && o.zero_x0) {
        // initial guess x0 = M(b) (FP64 application); kept only if it lowers the residual
        CG_TRY(fno::apply(c->net, s, c->N, 0, bp, c->chi32, (float)c->k0h, xp, nullptr));
        x0_learned = 1;
    }

    CycleProf cp;
    int it_prev = 0;
    const double nd = (double)n, esz_d = prec == 0 ? 16.0 : 8.0;

    // True residual r = b - A x (FP64) into V_0, the cycle decisions on the
    // device, and the copy of the state to the host.
    auto enqueue_begin = [&](cudaStream_t q) -> int {
        CG_LAUNCH(launch_rows_forward(0, a64, xs, nullptr, nullptr, GATE_NONE, q));
        CG_LAUNCH(launch_cols_convolve(0, a64, nullptr, GATE_NONE, q));
        CG_LAUNCH(launch_rows_inverse(0, 1, prec, a64, xs, nullptr, bp, fixed_vec(c->V), kp.npart, nullptr, GATE_NONE, q));
        CG_TRY(prof_mark(c, cp, CG_PHASE_RESIDUAL, -1, q));
        CG_LAUNCH(launch_cycle_begin(kp, nrb, q));
        CG_TRY(prof_mark(c, cp, CG_PHASE_SMALL, -1, q));
        CG_CU(cudaMemcpyAsync(c->st_host, c->st, sizeof(DevState), cudaMemcpyDeviceToHost, q));
        return CG_OK;
    };
    // One restart cycle: `steps` Arnoldi steps (launches after the device
    // stops the cycle return at once), back-solve and solution update.
    bool use_prec = learned;  // this cycle runs the learned preconditioner
    auto enqueue_cycle = [&](int steps, cudaStream_t q) -> int {
        for (int i = 0; i < steps; i++) {
            if (delayed) {
                // w = A u_k into V[k+1]; one dot pass; normalisation + Givens; one axpy pass
                CG_LAUNCH(launch_rows_forward(prec, ap, vk, nullptr, c->st, GATE_STOP, q));
                CG_LAUNCH(launch_cols_convolve(prec, ap, c->st, GATE_STOP, q));
                CG_LAUNCH(launch_rows_inverse(prec, 0, prec, ap, vk, nullptr, nullptr, vk1, nullptr, c->st, GATE_STOP, q));
                CG_TRY(prof_mark(c, cp, CG_PHASE_MATVEC, i, q));
                CG_LAUNCH(launch_dots2(prec, c->V, n, kp, ndot2, c->sms, q));
                CG_TRY(prof_mark(c, cp, CG_PHASE_DOTS, i, q));
                CG_LAUNCH(launch_dcgs2_step(kp, q));
                CG_TRY(prof_mark(c, cp, CG_PHASE_SMALL, i, q));
                CG_LAUNCH(launch_axpy2(prec, c->V, n, kp, nax2, c->sms, q));
                CG_TRY(prof_mark(c, cp, CG_PHASE_AXPY, i, q));
                continue;
            }
            if (use_prec) {
                // z_i = M(v_i) on the unnormalised stored vector (M is positively homogeneous)
                CG_TRY(fno::apply(c->net, q, c->N, prec, (const char *)c->V + (size_t)i * n * esz, c->chi32,
                                  (float)c->k0h, (char *)c->Z + (size_t)i * n * esz, &c->st->stop));
                CG_TRY(prof_mark(c, cp, CG_PHASE_PRECOND, i, q));
            }
            const VecSel &min = use_prec ? zk : vk;
            CG_LAUNCH(launch_rows_forward(prec, ap, min, kp.scale, c->st, GATE_STOP, q));
            CG_LAUNCH(launch_cols_convolve(prec, ap, c->st, GATE_STOP, q));
            CG_LAUNCH(launch_rows_inverse(prec, 0, prec, ap, min, kp.scale, nullptr, vk1, nullptr, c->st, GATE_STOP, q));
            CG_TRY(prof_mark(c, cp, CG_PHASE_MATVEC, i, q));
            CG_LAUNCH(launch_dots(prec, c->V, n, kp, vk1, kp.h1, 0, ndot, GATE_STOP, q));
            CG_TRY(prof_mark(c, cp, CG_PHASE_DOTS, i, q));
            CG_LAUNCH(launch_axpy(prec, prec, c->V, n, kp, kp.h1, -1.0, NJ_K_PLUS_1, vk1, 0, 1, nax, GATE_STOP, q));
            CG_TRY(prof_mark(c, cp, CG_PHASE_AXPY, i, q));
            CG_LAUNCH(launch_dots(prec, c->V, n, kp, vk1, kp.h2, 0, ndot, GATE_STOP, q));
            CG_TRY(prof_mark(c, cp, CG_PHASE_DOTS, i, q));
            CG_LAUNCH(launch_axpy(prec, prec, c->V, n, kp, kp.h2, -1.0, NJ_K_PLUS_1, vk1, 1, 1, nax, GATE_STOP, q));
            CG_TRY(prof_mark(c, cp, CG_PHASE_AXPY, i, q));
            CG_LAUNCH(launch_givens(kp, q));
            CG_TRY(prof_mark(c, cp, CG_PHASE_SMALL, i, q));
        }
        CG_LAUNCH(launch_backsolve(kp, q));
        CG_TRY(prof_mark(c, cp, CG_PHASE_SMALL, -1, q));
        CG_LAUNCH(launch_axpy(prec, 0, use_prec ? c->Z : c->V, n, kp, kp.y, 1.0, NJ_NCOL, xs, 0, 1, nax, GATE_NONE, q));
        CG_TRY(prof_mark(c, cp, CG_PHASE_UPDATE, -1, q));
        return CG_OK;
    };
    // s-step cycles: ceil(m / S) blocks of
    // S shifted matvecs, two block Gram-Schmidt passes and the Hessenberg /
    // Givens kernel, then the back-solve and the update
    bool ss_on = false;
    double2 shifts[SS_MAX];
    for (int i = 0; i < SS_MAX; i++) shifts[i] = make_double2(0.0, 0.0);
    // Long s-step cycles (restart above SS_REFRESH_MIN) are enqueued in segments
    // of SS_REFRESH_STEPS steps; after each, the Newton shifts become the
    // Leja-ordered Ritz values of the trailing SS_REFRESH_WINDOW columns of H.
    // The probe's shifts follow the outer spectrum that Arnoldi finds first; a
    // basis of thousands of vectors has left it behind, and with those shifts a
    // block's later vectors kept almost nothing outside the basis, so its
    // Cholesky failed and the cycle restarted (512^2, eps_r = 4, restart 4500:
    // 7 cycles and 12 000 steps without reaching 1e-10).  With the refresh the
    // first cycle runs 3981 steps (delayed CGS2: 3979) and a second of 1663
    // removes the 1e-8 its Hessenberg reconstruction left.  Each cycle starts
    // again from the probe's shifts.
    constexpr int SS_REFRESH_MIN = 256, SS_REFRESH_STEPS = 100, SS_REFRESH_WINDOW = 32;
    const bool ss_segments = m > SS_REFRESH_MIN;
    const int ss_nblk = S > 0 ? (m + S - 1) / S : 0;  // blocks of a full s-step cycle
    double2 shifts0[SS_MAX];
    for (int i = 0; i < SS_MAX; i++) shifts0[i] = make_double2(0.0, 0.0);
    const int nss = sstep_blocks(c->sms, n);
    auto enqueue_cycle_ss = [&](cudaStream_t q, int b0, int b1, bool finish) -> int {
        if (b0 == 0) {
            CG_LAUNCH(launch_ss_norm0(prec, c->V, n, kp, q));
            CG_TRY(prof_mark(c, cp, CG_PHASE_SMALL, -1, q));
        }
        // The Hessenberg / Givens kernel of block b (one block of threads) runs on a
        // side stream while block b + 1's Newton chain runs: the chain addresses its
        // rows absolutely (block b starts at column b S) instead of through st->k,
        // and the join precedes block b + 1's dot pass, the first kernel that reads
        // what the Hessenberg kernel writes.  A cycle that the Hessenberg kernel
        // stops lets the chain finish on rows the cycle no longer uses; every later
        // kernel sees the stop.  Profiled cycles keep one stream (exact phase times).
        const bool overlap = !c->prof;
        if (overlap && !c->side_stream) {
            CG_CU(cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking));
            CG_CU(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
            CG_CU(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
        }
        bool pending = false;
        for (int b = b0; b < b1 && b * S < m; b++) {
            const bool last_block = (b + 1) * S >= m || b + 1 >= b1;
            // Newton chain w_{i+1} = (A - theta_i) w_i: the inverse row pass of each
            // matvec but the last also runs the next one's forward row pass
            const bool chain = !o.transpose;
            for (int i = 0; i < S; i++) {
                VecSel vin = vk, vout = vk;
                vin.koff = b * S + i;
                vout.koff = b * S + i + 1;
                vin.abs = vout.abs = 1;
                if (i == 0 || !chain) CG_LAUNCH(launch_rows_forward(prec, ap, vin, nullptr, c->st, GATE_STOP, q));
                CG_LAUNCH(launch_cols_convolve(prec, ap, c->st, GATE_STOP, q));
                if (chain && i + 1 < S)
                    CG_LAUNCH(launch_rows_inv_fwd(prec, ap, vin, vout, c->st, GATE_STOP, q, shifts[i]));
                else
                    CG_LAUNCH(launch_rows_inverse(prec, 0, prec, ap, vin, nullptr, nullptr, vout, nullptr, c->st,
                                                  GATE_STOP, q, shifts[i]));
            }
            CG_TRY(prof_mark(c, cp, CG_PHASE_MATVEC, b * S, q));
            if (pending) {
                CG_CU(cudaStreamWaitEvent(q, c->ev_join, 0));
                pending = false;
            }
            for (int pass = 0; pass < 2; pass++) {
                // the dot pass's last block also runs the pass's Cholesky
                CG_LAUNCH(launch_ss_dots(prec, c->V, n, kp, S, c->sms, pass, q));
                CG_TRY(prof_mark(c, cp, CG_PHASE_DOTS, b * S, q));
                CG_LAUNCH(launch_ss_update(prec, c->V, n, kp, S, c->sms, pass, q));
                CG_TRY(prof_mark(c, cp, CG_PHASE_AXPY, b * S, q));
            }
            if (overlap && !last_block) {
                CG_CU(cudaEventRecord(c->ev_fork, q));
                CG_CU(cudaStreamWaitEvent(c->side_stream, c->ev_fork, 0));
                CG_LAUNCH(launch_ss_hess(kp, S, b * S, c->side_stream));
                CG_CU(cudaEventRecord(c->ev_join, c->side_stream));
                pending = true;
            } else {
                CG_LAUNCH(launch_ss_hess(kp, S, b * S, q));
                CG_TRY(prof_mark(c, cp, CG_PHASE_SMALL, b * S, q));
            }
        }
        if (!finish) return CG_OK;
        CG_LAUNCH(launch_backsolve(kp, q));
        CG_TRY(prof_mark(c, cp, CG_PHASE_SMALL, -1, q));
        CG_LAUNCH(launch_axpy(prec, 0, c->V, n, kp, kp.y, 1.0, NJ_NCOL, xs, 0, 1, nax, GATE_NONE, q));
        CG_TRY(prof_mark(c, cp, CG_PHASE_UPDATE, -1, q));
        return CG_OK;
    };
    // Fallback when the probe before the solve gave no shifts: the solve's first
    // cycle runs delayed CGS2 and its Hessenberg (unrotated in Hm) gives them,
    // Leja-ordered Ritz values; s-step stays off when that cycle had fewer than S columns.
    auto setup_shifts = [&](int ncol1) -> int {
        if (ncol1 < S) return CG_OK;
        const int ld = c->mcap + 1;
        std::vector<double2> hm((size_t)ncol1 * ld);
        CG_CU(cudaMemcpyAsync(hm.data(), kp.Hm, sizeof(double2) * hm.size(), cudaMemcpyDeviceToHost, s));
        CG_CU(cudaStreamSynchronize(s));
        const std::vector<std::complex<double>> ritz = hessenberg_eigenvalues(hm, ncol1, ld);
        for (const auto &z : ritz)
            if (!std::isfinite(z.real()) || !std::isfinite(z.imag())) return CG_OK;
        const std::vector<std::complex<double>> th = leja_points(ritz, S);
        for (int i = 0; i < S; i++) shifts[i] = make_double2(th[i].real(), th[i].imag());
        for (int i = 0; i < SS_MAX; i++) shifts0[i] = shifts[i];
        // the Hessenberg kernel reads them from the scratch (offset of SsLayout::Th)
        const long long M1 = c->mcap + 1;
        const long long th_off = 3 * M1 * SS_MAX + 3 * SS_MAX * SS_MAX;
        CG_CU(cudaMemcpyAsync(kp.ss + th_off, shifts, sizeof(double2) * SS_MAX, cudaMemcpyHostToDevice, s));
        CG_CU(cudaStreamSynchronize(s));
        ss_on = true;
        return CG_OK;
    };
    if (probe_ok) {
        for (int i = 0; i < SS_MAX; i++) shifts[i] = shifts0[i] = shifts_probe[i];
        // the Hessenberg kernel reads them from the scratch (offset of SsLayout::Th)
        const long long M1 = c->mcap + 1;
        const long long th_off = 3 * M1 * SS_MAX + 3 * SS_MAX * SS_MAX;
        CG_CU(cudaMemcpyAsync(kp.ss + th_off, shifts, sizeof(double2) * SS_MAX, cudaMemcpyHostToDevice, s));
        ss_on = true;
    }
    // Graph replay of [cycle + next residual/decisions] when nothing in it
    // changes between cycles (not while profiling, not with the network).
    // (flexible GMRES: plain cycles after the probe only)
    const bool graphs = !c->prof && !c->in_probe && graphs_enabled();
    unsigned char key[256];
    // key of the cycle about to be replayed (the scheme can change between cycles)
    auto make_key = [&]() {
        memset(key, 0, sizeof(key));
        struct K {
            int prec, delayed, m, transpose, ndot, nax, ndot2, nax2, nrb, mcap, var[2][3], ss, nss;
            long long n;
            const void *V, *x, *b, *st, *scale, *part;
            double2 shifts[SS_MAX];
        } kk;
        memset(&kk, 0, sizeof(kk));
        kk.prec = prec, kk.delayed = delayed, kk.m = m, kk.transpose = o.transpose, kk.ndot = ndot, kk.nax = nax;
        kk.ndot2 = ndot2, kk.nax2 = nax2, kk.nrb = nrb, kk.mcap = c->mcap, kk.n = n;
        memcpy(kk.var, c->var, sizeof(kk.var));
        kk.V = c->V, kk.x = xp, kk.b = bp, kk.st = c->st, kk.scale = kp.scale, kk.part = kp.part;
        kk.ss = ss_on ? S : 0;
        kk.nss = nss;
        if (ss_on) memcpy(kk.shifts, shifts, sizeof(shifts));
        static_assert(sizeof(K) <= sizeof(key), "graph key");
        memcpy(key, &kk, sizeof(kk));
    };
    auto launch_cycle_graph = [&]() -> int {
        make_key();
        if (!c->gexec || memcmp(c->gkey, key, sizeof(key)) != 0) {
            free_graph(c);
            if (!c->cap_stream) CG_CU(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
            cudaGraph_t g = nullptr;
            CG_CU(cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal));
            int e1 = ss_on ? enqueue_cycle_ss(c->cap_stream, 0, ss_nblk, true)
                           : enqueue_cycle(m + (delayed ? 1 : 0), c->cap_stream);
            int e2 = e1 == CG_OK ? enqueue_begin(c->cap_stream) : e1;
            cudaError_t ce = cudaStreamEndCapture(c->cap_stream, &g);
            if (e2 != CG_OK || ce != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                return e2 != CG_OK ? e2 : CG_ERR_CUDA;
            }
            ce = cudaGraphInstantiate(&c->gexec, g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) {
                c->gexec = nullptr;
                cudaGetLastError();
                return CG_ERR_CUDA;
            }
            memcpy(c->gkey, key, sizeof(key));
        }
        CG_CU(cudaGraphLaunch(c->gexec, s));
        return CG_OK;
    };

    if (cp.used == 0) CG_TRY(prof_mark(c, cp, -1, -1, s));
    CG_TRY(enqueue_begin(s));
    for (;;) {
        CG_CU(cudaEventRecord(c->ev, s));
        CG_CU(cudaEventSynchronize(c->ev));
        const DevState hs = *c->st_host;
        CG_TRY(prof_collect(c, cp, nd, esz_d, hs.it - it_prev + (delayed && !ss_on ? 1 : 0), delayed && !ss_on,
                            ss_on ? S : 0, ss_on && !o.transpose));
        const int cycle_steps = hs.it - it_prev;
        it_prev = hs.it;
        // the first cycle has ended and the second begun: its Hessenberg gives the shifts
        if (sstep && !ss_on && hs.cycles == 2 && hs.status == 0) CG_TRY(setup_shifts(std::min(cycle_steps, m)));
        if (x0_learned == 1 && hs.cycles == 1 && hs.status == 0 && !(hs.true_res < 1.0)) {
            // M(b) did not beat x0 = 0: restart from zero (the cycle counter and budget are unchanged
            // because no Arnoldi step ran)
            CG_CU(cudaMemsetAsync(xp, 0, bytes, s));
            x0_learned = 0;
            DevState h2 = hs;
            h2.cycles = 0;
            *c->st_host = h2;
            CG_CU(cudaMemcpyAsync(c->st, c->st_host, sizeof(DevState), cudaMemcpyHostToDevice, s));
            if (cp.used == 0) CG_TRY(prof_mark(c, cp, -1, -1, s));
            CG_TRY(enqueue_begin(s));
            continue;
        }
        if (learned && cycle_open) {
            const double dt = now_s() - cycle_t0;
            const double red = (cycle_res0 > 0.0 && hs.true_res > 0.0) ? log(cycle_res0 / hs.true_res) : 0.0;
            const double rate = dt > 0.0 ? red / dt : 0.0;
            if (last_prec) {
                rate_prec = rate;
                if (!(red > 0.0)) prec_failed = true;
            } else {
                rate_plain = rate;
            }
        }
        if (learned) {
            if (prec_failed) use_prec = false;
            else if (rate_prec < 0.0) use_prec = true;
            else if (rate_plain < 0.0) use_prec = false;
            else use_prec = rate_prec > rate_plain;
        }
        if (hs.status != 0) break;
        if (o.timeout_s > 0.0 && now_s() - t0 > o.timeout_s) {
            status = CG_ERR_TIMEOUT;
            break;
        }
        CG_TRY(prof_mark(c, cp, -1, -1, s));
        if (use_prec) prec_cycles++;
        cycle_open = true;
        last_prec = use_prec;
        cycle_t0 = now_s();
        cycle_res0 = hs.true_res;
        if (learned) {
            const bool d = want_delayed && !use_prec;
            if (d != delayed) CG_LAUNCH(launch_set_ortho(kp, d ? 0 : 1, s));
            delayed = d;
        }
        // s-step without probe shifts, first cycle: delayed CGS2 for the shifts, at most 64 steps when the
        // restart is long (an unrestarted solve would otherwise spend its whole
        // budget before the s-step blocks start); restarts up to 128 keep their
        // full first cycle, so GMRES(m) iterates are those of the other schemes
        const bool ss_probe = sstep && !ss_on;
        if (ss_probe) {
            int len = std::min(m <= 128 ? m : 64, o.max_iter - hs.it);
            CG_TRY(enqueue_cycle(len + 1, s));
            CG_TRY(prof_mark(c, cp, -1, -1, s));
            CG_TRY(enqueue_begin(s));
        } else if (graphs && !use_prec && !(learned && rate_plain < 0.0) && !(ss_on && ss_segments)) {
            CG_TRY(launch_cycle_graph());
        } else if (ss_on && ss_segments) {
            const long long th_off = 3 * (long long)(c->mcap + 1) * SS_MAX + 3 * SS_MAX * SS_MAX;  // SsLayout::Th
            for (int i = 0; i < SS_MAX; i++) shifts[i] = shifts0[i];
            CG_CU(cudaMemcpyAsync(kp.ss + th_off, shifts, sizeof(double2) * SS_MAX, cudaMemcpyHostToDevice, s));
            const int segb = (SS_REFRESH_STEPS + S - 1) / S;
            int b0 = 0;
            for (;;) {
                CG_TRY(enqueue_cycle_ss(s, b0, b0 + segb, false));
                b0 += segb;
                if (b0 >= ss_nblk) break;
                DevState sd;
                CG_CU(cudaMemcpyAsync(&sd, c->st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
                CG_CU(cudaStreamSynchronize(s));
                if (sd.stop) break;
                if (o.timeout_s > 0.0 && now_s() - t0 > o.timeout_s) {
                    // end the cycle at the finished columns (nothing is in flight); the
                    // check after the cycle then returns CG_ERR_TIMEOUT
                    const int one = 1;
                    CG_CU(cudaMemcpyAsync(reinterpret_cast<char *>(c->st) + offsetof(DevState, stop), &one, sizeof(int),
                                          cudaMemcpyHostToDevice, s));
                    break;
                }
                const int k = sd.k, W = std::min(SS_REFRESH_WINDOW, k);
                if (W >= S) {
                    const int ld = c->mcap + 1;
                    std::vector<double2> hw((size_t)W * W);
                    CG_CU(cudaMemcpy2DAsync(hw.data(), sizeof(double2) * W, kp.Hm + (size_t)(k - W) * ld + (k - W),
                                            sizeof(double2) * ld, sizeof(double2) * W, W, cudaMemcpyDeviceToHost, s));
                    CG_CU(cudaStreamSynchronize(s));
                    const std::vector<std::complex<double>> ritz = hessenberg_eigenvalues(hw, W, W);
                    bool fin = true;
                    for (const auto &z : ritz) fin = fin && std::isfinite(z.real()) && std::isfinite(z.imag());
                    if (fin) {
                        const std::vector<std::complex<double>> th = leja_points(ritz, S);
                        for (int i = 0; i < S; i++) shifts[i] = make_double2(th[i].real(), th[i].imag());
                        // the next segment's Hessenberg kernels read them there
                        CG_CU(cudaMemcpyAsync(kp.ss + th_off, shifts, sizeof(double2) * SS_MAX, cudaMemcpyHostToDevice, s));
                    }
                }
            }
            CG_TRY(enqueue_cycle_ss(s, ss_nblk, ss_nblk, true));  // the back-solve and the update
            CG_TRY(prof_mark(c, cp, -1, -1, s));
            CG_TRY(enqueue_begin(s));
        } else if (ss_on) {
            CG_TRY(enqueue_cycle_ss(s, 0, ss_nblk, true));
            CG_TRY(prof_mark(c, cp, -1, -1, s));
            CG_TRY(enqueue_begin(s));
        } else {
            int len = std::min(m, o.max_iter - hs.it);
            if (learned && (use_prec || rate_plain < 0.0)) len = std::min(len, LEARNED_CYCLE_STEPS);
            CG_TRY(enqueue_cycle(len + (delayed ? 1 : 0), s));
            CG_TRY(prof_mark(c, cp, -1, -1, s));
            CG_TRY(enqueue_begin(s));
        }
    }
    if (learned) CG_TRY(fno::check_error(c->net));

    const DevState hs = *c->st_host;
    if (status == CG_OK) {
        switch (hs.status) {
            case 1: status = CG_OK; break;
            case 2: status = o.fixed_iterations ? CG_OK : CG_ERR_NOT_CONVERGED; break;
            case 3: status = CG_ERR_BREAKDOWN; break;
            case 4: status = CG_ERR_NONFINITE; break;
            default: status = CG_ERR_CUDA; break;
        }
    }
    if (res_hist && res_hist_len > 0) {
        const int nh = std::min(res_hist_len, hs.it + 1);
        CG_CU(cudaMemcpyAsync(res_hist, kp.hist, sizeof(double) * nh, cudaMemcpyDeviceToHost, s));
    }
    if (!xd) CG_CU(cudaMemcpyAsync(x, xp, bytes, cudaMemcpyDeviceToHost, s));
    CG_CU(cudaStreamSynchronize(s));
    if (result) {
        result->status = status;
        result->iterations = hs.it;
        result->cycles = hs.cycles;
        result->rel_residual_estimate = hs.est;
        result->rel_residual_true = hs.true_res;
        result->seconds = now_s() - t0;
        result->preconditioned_cycles = prec_cycles;
        result->x0_learned = x0_learned;
    }
    return status;
}

int cugmres_fast_gmres(const cg_c64 *g_prep, const unsigned char *mask, cg_c64 *solution, float *actual_residual,
                       unsigned int *gmres_n, float tolerance, int *res_vs_tol, unsigned int maxiter, unsigned int N,
                       float chi_value, const cg_c64 *rhs, int precision) {
    if (!g_prep || !mask || !solution || N < 1 || maxiter < 1) return CG_ERR_INVALID;
    const size_t n = (size_t)N * N;
    int dev = 0;
    CG_CU(cudaGetDevice(&dev));
    // host copies of the inputs (pointers may be device memory, as in the reference)
    std::vector<unsigned char> hm(n);
    std::vector<cg_c64> hx(n), hb(n);
    if (is_device_ptr(mask)) CG_CU(cudaMemcpy(hm.data(), mask, n, cudaMemcpyDeviceToHost));
    else memcpy(hm.data(), mask, n);
    const bool sol_dev = is_device_ptr(solution);
    if (sol_dev) CG_CU(cudaMemcpy(hx.data(), solution, sizeof(cg_c64) * n, cudaMemcpyDeviceToHost));
    else memcpy(hx.data(), solution, sizeof(cg_c64) * n);
    if (rhs) {
        if (is_device_ptr(rhs)) CG_CU(cudaMemcpy(hb.data(), rhs, sizeof(cg_c64) * n, cudaMemcpyDeviceToHost));
        else memcpy(hb.data(), rhs, sizeof(cg_c64) * n);
    } else {
        // the reference's incident field exp(-i k row), CUDA_GMRES/GMRES_kernels.cuh:557-572
        const float k = (2 * 3.14f) / ((float)N / 6.f);
        for (unsigned int i = 0; i < N; i++) {
            const float arg = (float)(-(double)k * (double)i);
            for (unsigned int j = 0; j < N; j++) hb[(size_t)i * N + j] = {cosf(arg), sinf(arg)};
        }
    }
    std::vector<double> chi(n);
    for (size_t e = 0; e < n; e++) chi[e] = hm[e] ? (double)chi_value : 0.0;
    std::vector<cg_c128> b128(n), x128(n);
    for (size_t e = 0; e < n; e++) {
        b128[e] = {hb[e].re, hb[e].im};
        x128[e] = {hx[e].re, hx[e].im};
    }
    cg_ctx *c = nullptr;
    CG_TRY(cugmres_create(&c, dev));
    int s = cugmres_set_operator_circulant(c, (int)N, g_prep, chi.data(), 1.0);
    std::vector<double> hist(maxiter + 1, 0.0);
    cg_result r;
    memset(&r, 0, sizeof(r));
    if (s == CG_OK) {
        cg_opts o;
        cugmres_default_opts(&o);
        o.restart = (int)maxiter;
        o.max_iter = (int)maxiter;
        o.tol = tolerance;
        o.fixed_iterations = 1;
        o.givens = CG_GIVENS_REFERENCE;
        o.precision = precision;
        o.inner_tol = 0.0;
        s = cugmres_solve(c, b128.data(), x128.data(), &o, hist.data(), (int)maxiter + 1, &r);
    }
    if (s == CG_OK) {
        double nb = 0.0;
        for (size_t e = 0; e < n; e++) nb += b128[e].re * b128[e].re + b128[e].im * b128[e].im;
        nb = sqrt(nb);
        std::vector<float> res(maxiter + 1, 0.f);
        for (int i = 0; i <= r.iterations && i <= (int)maxiter; i++) res[i] = (float)(hist[i] * nb);
        for (size_t e = 0; e < n; e++) hx[e] = {(float)x128[e].re, (float)x128[e].im};
        if (sol_dev) s = cuerr(cudaMemcpy(solution, hx.data(), sizeof(cg_c64) * n, cudaMemcpyHostToDevice));
        else memcpy(solution, hx.data(), sizeof(cg_c64) * n);
        if (actual_residual) {
            if (is_device_ptr(actual_residual))
                s = cuerr(cudaMemcpy(actual_residual, res.data(), sizeof(float) * (maxiter + 1), cudaMemcpyHostToDevice));
            else memcpy(actual_residual, res.data(), sizeof(float) * (maxiter + 1));
        }
        if (gmres_n) *gmres_n = (unsigned int)r.iterations;
        if (res_vs_tol) *res_vs_tol = (r.iterations > 0 ? res[r.iterations] : res[0]) > tolerance;
    }
    cugmres_destroy(c);
    return s;
}

}  // extern "C"
