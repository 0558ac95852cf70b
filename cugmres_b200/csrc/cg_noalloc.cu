// Allocation-free operator application, cugmres_matvec_noalloc.
//
// Some callers cannot allocate device memory: a host application whose GPU
// memory is entirely owned by its own pool allocator (and which does not let a
// plug-in grow or fragment it), or a latency-critical loop that cannot afford
// the implicit device-wide synchronisation of cudaMalloc / cudaFree.  For them
// this file offers one entry point that computes y = A x (FP64) from the
// Green's block, the contrast and x without any allocation: every
// intermediate buffer lives in the file-scope device array g_noalloc_scratch
// below, whose size fixes the largest grid it accepts (N <= 256, so
// L <= 512).  Every GPU that loads the library keeps this array (about 7.9 MB)
// until the process exits.
//
// Properties a caller must know:
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current); make
//     that first call before any stream capture;
//   * that address is kept for the life of the process: the library must not
//     outlive a cudaDeviceReset (or any other teardown of the device's primary
//     context), after which the kept address would be stale;
//   * all calls on a device share the one array, so calls whose work overlaps
//     on the GPU (different streams, or different host threads) race; serialise
//     them on one stream;
//   * each call overwrites every scratch region it reads, so nothing depends on
//     what a previous call left there;
//   * the call only enqueues work on `stream` and returns; y is valid once the
//     stream has reached that point.
#include <mutex>

#include "../../include/cugmres.h"
#include "cg_common.cuh"
#include "cg_fft.cuh"
#include "cg_internal.h"

namespace {

constexpr int NA_MAX_N = CUGMRES_NOALLOC_MAX_N;
constexpr int NA_MAX_L = 2 * NA_MAX_N;  // embedding of the largest accepted grid
constexpr size_t na_align(size_t v) { return (v + 255) & ~(size_t)255; }
constexpr size_t NA_OFF_FULL = 0;                                                       // L x L spectrum
constexpr size_t NA_OFF_QUARTER = na_align(NA_OFF_FULL + (size_t)NA_MAX_L * NA_MAX_L * sizeof(double2));
constexpr size_t NA_OFF_T = na_align(NA_OFF_QUARTER + (size_t)(NA_MAX_L / 2 + 1) * (NA_MAX_L / 2 + 1) * sizeof(double2));
constexpr size_t NA_OFF_C = na_align(NA_OFF_T + (size_t)NA_MAX_N * NA_MAX_L * sizeof(double2));
constexpr size_t NA_OFF_TW = na_align(NA_OFF_C + (size_t)NA_MAX_N * NA_MAX_N * sizeof(double));
constexpr size_t NA_BYTES = na_align(NA_OFF_TW + (size_t)4 * NA_MAX_L * sizeof(double2));

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
void *g_na_ptr[NA_MAX_DEVICES] = {};

// Device address of g_noalloc_scratch on the current device (looked up once).
int na_scratch(int dev, unsigned char **out) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return CG_ERR_CUDA;
        }
        g_na_ptr[dev] = p;
    }
    *out = (unsigned char *)g_na_ptr[dev];
    return CG_OK;
}

// True when p is device (or managed) memory that belongs to device `dev`; a
// pointer into another GPU's memory is refused, since the kernels would read it
// over the peer link (or fault without peer access).
bool na_on_device(const void *p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return false;
    return a.device == dev;
}

// the four per-stage twiddle tables of cg_fft.cuh (16- and 8-point plans,
// forward and inverse), 4 L entries
__global__ void k_na_twiddles(double2 *tw, int L) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 4 * L; e += gridDim.x * blockDim.x) {
        const int t = e / L, i = e % L;
        const int m = cg::twiddle_exponent(L, t < 2 ? 16 : 8, i);
        double s = 0.0, c = 0.0;
        if (m >= 0) sincospi(2.0 * (double)m / (double)L, &s, &c);
        tw[e] = make_double2(c, (t & 1) ? s : -s);
    }
}

// even circulant embedding of the N x N block into L x L
__global__ void k_na_embed(const double2 *__restrict__ g, double2 *__restrict__ full, int N, int L) {
    const int tot = L * L;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += gridDim.x * blockDim.x) {
        const int i = e / L, j = e % L;
        const int di = i <= L - i ? i : L - i;
        const int dj = j <= L - j ? j : L - j;
        full[e] = (di < N && dj < N) ? g[di * N + dj] : make_double2(0.0, 0.0);
    }
}

// quarter of the (even) spectrum with 1/L^2 folded in; contrast c = scale * chi
__global__ void k_na_prepare(const double2 *__restrict__ full, double2 *__restrict__ quarter, int L,
                             const double *__restrict__ chi, double scale, double *__restrict__ c, int n) {
    const int Lq = L / 2 + 1;
    const double inv = 1.0 / ((double)L * (double)L);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Lq * Lq; e += gridDim.x * blockDim.x) {
        const double2 v = full[(e % Lq) * L + (e / Lq)];  // column-major quarter
        quarter[e] = make_double2(v.x * inv, v.y * inv);
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) c[e] = chi[e] * scale;
}

}  // namespace

extern "C" int cugmres_matvec_noalloc(int N, const cg_c128 *g_block, const double *chi, double chi_scale,
                                      const cg_c128 *x, cg_c128 *y, void *stream) {
    if (N < 1 || !g_block || !chi || !x || !y || !isfinite(chi_scale)) return CG_ERR_INVALID;
    if (N > NA_MAX_N) return CG_ERR_INVALID;  // beyond the fixed scratch: use cugmres_matvec
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CG_ERR_CUDA;
    if (!na_on_device(g_block, dev) || !na_on_device(chi, dev) || !na_on_device(x, dev) || !na_on_device(y, dev))
        return CG_ERR_INVALID;
    int L = 16;
    while (L < 2 * N - 1) L *= 2;
    unsigned char *base = nullptr;
    int st = na_scratch(dev, &base);
    if (st != CG_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    double2 *full = (double2 *)(base + NA_OFF_FULL);
    double2 *quarter = (double2 *)(base + NA_OFF_QUARTER);
    double2 *T = (double2 *)(base + NA_OFF_T);
    double *c = (double *)(base + NA_OFF_C);
    double2 *tw = (double2 *)(base + NA_OFF_TW);

    k_na_twiddles<<<(4 * L + 255) / 256, 256, 0, s>>>(tw, L);
    k_na_embed<<<(L * L + 255) / 256, 256, 0, s>>>((const double2 *)g_block, full, N, L);
    if (cudaGetLastError() != cudaSuccess) return CG_ERR_CUDA;
    if (cg::launch_fft2d_full_fp64(L, full, tw, s) != 0) return CG_ERR_CUDA;
    const int nq = (L / 2 + 1) * (L / 2 + 1);
    k_na_prepare<<<((nq > N * N ? nq : N * N) + 255) / 256, 256, 0, s>>>(full, quarter, L, chi, chi_scale, c, N * N);
    if (cudaGetLastError() != cudaSuccess) return CG_ERR_CUDA;

    cg::MatvecArgs a;
    a.N = N;
    a.L = L;
    a.vfwd = a.vcols = a.vinv = 0;
    a.gq = quarter;
    a.cdiag = c;
    a.tw = tw;
    a.T = T;
    cg::VecSel xs, ys;
    xs.base = (void *)x;
    xs.stride = 0;
    xs.koff = 0;
    ys.base = (void *)y;
    ys.stride = 0;
    ys.koff = 0;
    if (cg::launch_rows_forward(0, a, xs, nullptr, nullptr, cg::GATE_NONE, s) != 0) return CG_ERR_CUDA;
    if (cg::launch_cols_convolve(0, a, nullptr, cg::GATE_NONE, s) != 0) return CG_ERR_CUDA;
    if (cg::launch_rows_inverse(0, 0, 0, a, xs, nullptr, nullptr, ys, nullptr, nullptr, cg::GATE_NONE, s) != 0)
        return CG_ERR_CUDA;
    return CG_OK;
}
