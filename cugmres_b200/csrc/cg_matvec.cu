// The BTTB operator y = x - G (c .* x), c = k0^2 chi, applied by circulant
// embedding into an L x L grid (L >= 2N-1, power of two) in three HBM passes.
//
// Reference behaviour (CUDA_GMRES/Fast_matvec.cuh:1-28 with
// GMRES_kernels.cuh:98-121,151-167,286-303): pad c.*x into a zero (2N-1)^2 array,
// cuFFT forward, multiply by the spectrum, cuFFT inverse, crop the N x N corner
// and subtract from x -- five kernels, each followed by a device sync.
//
// Here:
//   pass 1  k_rows_forward   rows 0..N-1 only: load x and c, scale, zero-pad in
//                            registers, forward row FFT, store T[N][L].
//   pass 2  k_cols_convolve  per column: forward column FFT (upper half of the
//                            input is zero), multiply by the spectrum, inverse
//                            column FFT, store only rows 0..N-1 back into T.
// Twiddle tables hold 2L entries: exp(-2 pi i m/L) then its conjugate, so the
// inverse transform reads different addresses from the forward one (otherwise
// the compiler keeps the forward twiddles live across the column convolution).
//   pass 3  k_rows_inverse   inverse row FFT, crop to the first N columns and
//                            finish: y = s x - conv  (matvec)  or
//                            r = b - x + conv (residual), with ||y||^2 partials.
// The spectrum is even in both axes for the reference's kernel and for the
// GFIEM kernel (G depends on |d1|, |d2|), so only its quarter
// (L/2+1) x (L/2+1) is stored and read; the 1/L^2 normalisation is folded into it.
#include "cg_fft.cuh"
#include "cg_internal.h"

namespace cg {

template <typename C> struct PrecOf;
template <> struct PrecOf<double2> { static const int value = 0; };
template <> struct PrecOf<float2> { static const int value = 1; };

static __device__ __forceinline__ bool gated(const DevState *st, int gate) {
    return gate == GATE_STOP && st != nullptr && st->stop != 0;
}

static __device__ __forceinline__ long long sel_index(const DevState *st, int koff) {
    return st ? (long long)(st->k + koff) : 0;
}

template <int L> struct RowCfg {
    static constexpr int TPR = Plan<L>::TPR;
    static constexpr int RPC = (TPR >= 256) ? 1 : 256 / TPR;
    static constexpr int THREADS = RPC * TPR;
};

// Column blocks: 256 threads for FP64 (16 complex doubles per thread need
// more than the 128 registers a 512-thread block allows), 512 for FP32.
template <int L, int ESZ> struct ColCfg {
    static constexpr int TPR = Plan<L>::TPR;
    static constexpr int TARGET = ESZ >= 16 ? 256 : 512;
    static constexpr int CPB0 = (TPR >= TARGET) ? 1 : TARGET / TPR;
    static constexpr int CPB = CPB0 > L ? L : CPB0;
    static constexpr int THREADS = CPB * TPR;
    // columns interleaved element by element: element i of column c at sm[pad(i) * CPB + c]
    static constexpr int SMEM_ELEMS = Plan<L>::SMEM_ELEMS * CPB;
};

// ---------------------------------------------------------------- pass 1
template <typename C, int L>
__global__ void __launch_bounds__(RowCfg<L>::THREADS)
k_rows_forward(VecSel xs, const double *__restrict__ xscale, const typename real_of<C>::type *__restrict__ cdiag,
               C *__restrict__ T, const C *__restrict__ tw, int N, const DevState *st, int gate) {
    typedef typename real_of<C>::type R;
    typedef Plan<L> P;
    constexpr int E = P::E, TPR = P::TPR;
    if (gated(st, gate)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lr = threadIdx.x / TPR, t = threadIdx.x % TPR;
    C *sm = reinterpret_cast<C *>(smraw) + lr * P::SMEM_ELEMS;
    const int row = blockIdx.x * RowCfg<L>::RPC + lr;
    const long long ks = sel_index(st, xs.koff);
    const C *x = reinterpret_cast<const C *>(xs.base) + ks * xs.stride;
    const R s = xscale ? (R)xscale[ks] : (R)1;
    C reg[E];
    const bool live = row < N;
    const size_t rb = (size_t)row * (size_t)N;
#pragma unroll
    for (int p = 0; p < E; p++) {
        const int idx = t + p * TPR;
        reg[p] = czero<C>();
        if (p < E / 2 && live && idx < N) {
            const C v = x[rb + idx];
            const R c = cdiag[rb + idx] * s;
            reg[p] = cscale(v, c);
        }
    }
    fft_run<L, false, true>(reg, sm, tw, t);
    if (live) {
        C *out = T + (size_t)row * L;
#pragma unroll
        for (int p = 0; p < E; p++) out[t + p * TPR] = reg[p];
    }
}

// ---------------------------------------------------------------- pass 2
template <typename C, int L>
#ifndef CG_COL_MINB
#define CG_COL_MINB 1
#endif
__global__ void __launch_bounds__(ColCfg<L, sizeof(C)>::THREADS, CG_COL_MINB)
k_cols_convolve(C *__restrict__ T, const C *__restrict__ gq, const C *__restrict__ tw, int N, const DevState *st,
                int gate) {
    typedef Plan<L> P;
    typedef ColCfg<L, sizeof(C)> Q;
    constexpr int E = P::E, TPR = P::TPR, CPB = Q::CPB;
    if (gated(st, gate)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int cl = threadIdx.x % CPB, t = threadIdx.x / CPB;
    C *sm = reinterpret_cast<C *>(smraw) + cl;
    // neighbouring blocks take mirrored column tiles so they share quarter-spectrum columns in L2
    const int ntiles = L / CPB;
    const int b = blockIdx.x;
    const int tile = (b & 1) ? (ntiles - 1 - (b >> 1)) : (b >> 1);
    const int col = tile * CPB + cl;
    C reg[E];
#pragma unroll
    for (int p = 0; p < E; p++) {
        const int k = t + p * TPR;
        reg[p] = czero<C>();
        if (p < E / 2 && k < N) reg[p] = T[(size_t)k * L + col];
    }
    fft_run<L, false, true, CPB>(reg, sm, tw, t);
    const int Lq = L / 2 + 1;
    const int qc = col <= L / 2 ? col : L - col;
#pragma unroll
    for (int p = 0; p < E; p++) {
        const int k1 = t + p * TPR;
        const int qr = k1 <= L / 2 ? k1 : L - k1;
        reg[p] = cmul(reg[p], __ldg(gq + (size_t)qr * Lq + qc));
    }
    fft_run<L, true, false, CPB>(reg, sm, tw + L, t);
#pragma unroll
    for (int p = 0; p < E / 2; p++) {
        const int k = t + p * TPR;
        if (k < N) T[(size_t)k * L + col] = reg[p];
    }
}

// ---------------------------------------------------------------- pass 3
template <typename C, typename CO, int L, int MODE>
__global__ void __launch_bounds__(RowCfg<L>::THREADS)
k_rows_inverse(const C *__restrict__ T, VecSel xs, const double *__restrict__ xscale, const C *__restrict__ bvec,
               VecSel ys, double *__restrict__ npart, const C *__restrict__ tw, int N, const DevState *st, int gate) {
    typedef typename real_of<C>::type R;
    typedef typename real_of<CO>::type RO;
    typedef Plan<L> P;
    constexpr int E = P::E, TPR = P::TPR;
    if (gated(st, gate)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double wsum[RowCfg<L>::THREADS / 32];
    const int lr = threadIdx.x / TPR, t = threadIdx.x % TPR;
    C *sm = reinterpret_cast<C *>(smraw) + lr * P::SMEM_ELEMS;
    const int row = blockIdx.x * RowCfg<L>::RPC + lr;
    const bool live = row < N;
    C reg[E];
    if (live) {
        const C *in = T + (size_t)row * L;
#pragma unroll
        for (int p = 0; p < E; p++) reg[p] = in[t + p * TPR];
    } else {
#pragma unroll
        for (int p = 0; p < E; p++) reg[p] = czero<C>();
    }
    fft_run<L, true, false>(reg, sm, tw + L, t);
    const long long kx = sel_index(st, xs.koff);
    const long long ky = sel_index(st, ys.koff);
    const C *x = reinterpret_cast<const C *>(xs.base) + kx * xs.stride;
    CO *y = reinterpret_cast<CO *>(ys.base) + ky * ys.stride;
    const R s = xscale ? (R)xscale[kx] : (R)1;
    double acc = 0.0;
    if (live) {
        const size_t rb = (size_t)row * (size_t)N;
#pragma unroll
        for (int p = 0; p < E / 2; p++) {
            const int idx = t + p * TPR;
            if (idx < N) {
                const C xv = x[rb + idx];
                C o;
                if (MODE == 0) {
                    o = csub(cscale(xv, s), reg[p]);
                } else {
                    o = cadd(csub(bvec[rb + idx], xv), reg[p]);
                }
                CO oo;
                oo.x = (RO)o.x;
                oo.y = (RO)o.y;
                y[rb + idx] = oo;
                acc += (double)o.x * (double)o.x + (double)o.y * (double)o.y;
            }
        }
    }
    if (npart) {
        acc = warp_sum(acc);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int w = 0; w < RowCfg<L>::THREADS / 32; w++) tot += wsum[w];
            npart[blockIdx.x] = tot;
        }
    }
}

// ------------------------------------------------- full transforms (setup)
template <int L>
__global__ void __launch_bounds__(RowCfg<L>::THREADS)
k_rows_fft_full(double2 *__restrict__ A, const double2 *__restrict__ tw) {
    typedef Plan<L> P;
    constexpr int E = P::E, TPR = P::TPR;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lr = threadIdx.x / TPR, t = threadIdx.x % TPR;
    double2 *sm = reinterpret_cast<double2 *>(smraw) + lr * P::SMEM_ELEMS;
    const int row = blockIdx.x * RowCfg<L>::RPC + lr;
    const bool live = row < L;
    double2 reg[E];
#pragma unroll
    for (int p = 0; p < E; p++) reg[p] = live ? A[(size_t)row * L + t + p * TPR] : czero<double2>();
    fft_run<L, false, false>(reg, sm, tw, t);
    if (live) {
#pragma unroll
        for (int p = 0; p < E; p++) A[(size_t)row * L + t + p * TPR] = reg[p];
    }
}

template <int L>
__global__ void __launch_bounds__(ColCfg<L, 16>::THREADS)
k_cols_fft_full(double2 *__restrict__ A, const double2 *__restrict__ tw) {
    typedef Plan<L> P;
    typedef ColCfg<L, 16> Q;
    constexpr int E = P::E, TPR = P::TPR, CPB = Q::CPB;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int cl = threadIdx.x % CPB, t = threadIdx.x / CPB;
    double2 *sm = reinterpret_cast<double2 *>(smraw) + cl;
    const int col = blockIdx.x * CPB + cl;
    double2 reg[E];
#pragma unroll
    for (int p = 0; p < E; p++) reg[p] = A[(size_t)(t + p * TPR) * L + col];
    fft_run<L, false, false, CPB>(reg, sm, tw, t);
#pragma unroll
    for (int p = 0; p < E; p++) A[(size_t)(t + p * TPR) * L + col] = reg[p];
}

// ---------------------------------------------------------------- launchers
template <typename K> static int set_smem(K kern, size_t bytes) {
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return (int)e;
    }
    return 0;
}

template <typename C, int L>
static int rows_forward_t(const MatvecArgs &a, VecSel x, const double *xs, const DevState *st, int gate,
                          cudaStream_t s) {
    typedef typename real_of<C>::type R;
    const size_t smem = (size_t)RowCfg<L>::RPC * Plan<L>::SMEM_ELEMS * sizeof(C);
    auto kern = k_rows_forward<C, L>;
    int e = set_smem(kern, smem);
    if (e) return e;
    const int grid = (a.N + RowCfg<L>::RPC - 1) / RowCfg<L>::RPC;
    kern<<<grid, RowCfg<L>::THREADS, smem, s>>>(x, xs, (const R *)a.cdiag, (C *)a.T, (const C *)a.tw, a.N, st, gate);
    return (int)cudaGetLastError();
}

template <typename C, int L>
static int cols_convolve_t(const MatvecArgs &a, const DevState *st, int gate, cudaStream_t s) {
    typedef ColCfg<L, sizeof(C)> Q;
    const size_t smem = (size_t)Q::SMEM_ELEMS * sizeof(C);
    auto kern = k_cols_convolve<C, L>;
    int e = set_smem(kern, smem);
    if (e) return e;
    const int grid = L / Q::CPB;
    kern<<<grid, Q::THREADS, smem, s>>>((C *)a.T, (const C *)a.gq, (const C *)a.tw, a.N, st, gate);
    return (int)cudaGetLastError();
}

template <typename C, typename CO, int L, int MODE>
static int rows_inverse_t(const MatvecArgs &a, VecSel x, const double *xs, const void *b, VecSel y, double *npart,
                          const DevState *st, int gate, cudaStream_t s) {
    const size_t smem = (size_t)RowCfg<L>::RPC * Plan<L>::SMEM_ELEMS * sizeof(C);
    auto kern = k_rows_inverse<C, CO, L, MODE>;
    int e = set_smem(kern, smem);
    if (e) return e;
    const int grid = (a.N + RowCfg<L>::RPC - 1) / RowCfg<L>::RPC;
    kern<<<grid, RowCfg<L>::THREADS, smem, s>>>((const C *)a.T, x, xs, (const C *)b, y, npart, (const C *)a.tw, a.N,
                                                 st, gate);
    return (int)cudaGetLastError();
}

template <int L> static int fft2d_full_t(double2 *A, const double2 *tw, cudaStream_t s) {
    size_t smem = (size_t)RowCfg<L>::RPC * Plan<L>::SMEM_ELEMS * sizeof(double2);
    auto kr = k_rows_fft_full<L>;
    int e = set_smem(kr, smem);
    if (e) return e;
    kr<<<(L + RowCfg<L>::RPC - 1) / RowCfg<L>::RPC, RowCfg<L>::THREADS, smem, s>>>(A, tw);
    e = (int)cudaGetLastError();
    if (e) return e;
    typedef ColCfg<L, 16> Q;
    smem = (size_t)Q::SMEM_ELEMS * sizeof(double2);
    auto kc = k_cols_fft_full<L>;
    e = set_smem(kc, smem);
    if (e) return e;
    kc<<<L / Q::CPB, Q::THREADS, smem, s>>>(A, tw);
    return (int)cudaGetLastError();
}

#define CG_FOR_EACH_L(X) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)

int fft_supported(int L) {
    switch (L) {
#define CASE(LL) case LL:
        CG_FOR_EACH_L(CASE)
#undef CASE
        return 1;
        default: return 0;
    }
}

int rows_per_block(int prec, int L) {
    (void)prec;
    switch (L) {
#define CASE(LL) \
    case LL: return RowCfg<LL>::RPC;
        CG_FOR_EACH_L(CASE)
#undef CASE
        default: return 1;
    }
}

int launch_rows_forward(int prec, const MatvecArgs &a, VecSel x, const double *xs, const DevState *st, int gate,
                        cudaStream_t s) {
    switch (a.L) {
#define CASE(LL)                                                                           \
    case LL:                                                                               \
        return prec == 0 ? rows_forward_t<double2, LL>(a, x, xs, st, gate, s)             \
                         : rows_forward_t<float2, LL>(a, x, xs, st, gate, s);
        CG_FOR_EACH_L(CASE)
#undef CASE
        default: return -1;
    }
}

int launch_cols_convolve(int prec, const MatvecArgs &a, const DevState *st, int gate, cudaStream_t s) {
    switch (a.L) {
#define CASE(LL)                                                                                      \
    case LL:                                                                                          \
        return prec == 0 ? cols_convolve_t<double2, LL>(a, st, gate, s) : cols_convolve_t<float2, LL>(a, st, gate, s);
        CG_FOR_EACH_L(CASE)
#undef CASE
        default: return -1;
    }
}

int launch_rows_inverse(int prec, int mode, int out_prec, const MatvecArgs &a, VecSel x, const double *xs,
                        const void *b, VecSel y, double *npart, const DevState *st, int gate, cudaStream_t s) {
    switch (a.L) {
#define CASE(LL)                                                                                         \
    case LL:                                                                                             \
        if (prec == 0) {                                                                                 \
            if (mode == 0)                                                                               \
                return rows_inverse_t<double2, double2, LL, 0>(a, x, xs, b, y, npart, st, gate, s);      \
            return out_prec == 0 ? rows_inverse_t<double2, double2, LL, 1>(a, x, xs, b, y, npart, st, gate, s) \
                                 : rows_inverse_t<double2, float2, LL, 1>(a, x, xs, b, y, npart, st, gate, s); \
        }                                                                                                \
        if (mode == 0) return rows_inverse_t<float2, float2, LL, 0>(a, x, xs, b, y, npart, st, gate, s); \
        return rows_inverse_t<float2, float2, LL, 1>(a, x, xs, b, y, npart, st, gate, s);
        CG_FOR_EACH_L(CASE)
#undef CASE
        default: return -1;
    }
}

int launch_fft2d_full_fp64(int L, double2 *A, const double2 *tw, cudaStream_t s) {
    switch (L) {
#define CASE(LL) \
    case LL: return fft2d_full_t<LL>(A, tw, s);
        CG_FOR_EACH_L(CASE)
#undef CASE
        default: return -1;
    }
}

}  // namespace cg
