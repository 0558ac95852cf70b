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
//   pass 3  k_rows_inverse   inverse row FFT, crop to the first N columns and
//                            finish: y = s x - conv  (matvec)  or
//                            r = b - x + conv (residual), with ||y||^2 partials.
// The spectrum is even in both axes for the reference's kernel and for the
// GFIEM kernel (G depends on |d1|, |d2|), so only its quarter
// (L/2+1) x (L/2+1) is stored and read, column-major (Gq[qc][qr]) so that the
// column pass reads it along its columns; the 1/L^2 normalisation is folded into it.
// Twiddle tables (cg_fft.cuh) hold 4L entries: per-stage forward and inverse
// tables of the 16- and 8-point plans.  The inverse transform reads different
// addresses from the forward one (otherwise the compiler keeps the forward
// twiddles live across the column convolution).
//
// Launch shapes (points per thread, threads per block, resident blocks per SM
// requested from the compiler, pipelined column pass) are template parameters;
// the MvShape variants 0..7 are instantiated for L >= 128 and the autotuner in cg_api.cu picks one
// per (precision, L); smaller L always use variant 0.
#include "cg_fft.cuh"
#include "cg_internal.h"

namespace cg {

static __device__ __forceinline__ bool gated(const DevState *st, int gate) {
    return gate == GATE_STOP && st != nullptr && st->stop != 0;
}

static __device__ __forceinline__ long long sel_index(const DevState *st, const VecSel &v) {
    if (v.abs) return (long long)v.koff;
    return st ? (long long)(st->k + v.koff) : 0;
}

// E: points per thread; ROWT: target threads per row block; COLT64 / COLT32:
// target threads per column block in FP64 / FP32; MINB: resident blocks per SM
// requested from the compiler (bounds the registers per thread); PIPE: the
// column pass is the persistent, double-buffered k_cols_convolve_pipe.
template <int E_, int ROWT_, int COLT64_, int COLT32_, int MINB_, int PIPE_ = 0> struct MvShape {
    static constexpr int E = E_, ROWT = ROWT_, COLT64 = COLT64_, COLT32 = COLT32_, MINB = MINB_, PIPE = PIPE_;
};
typedef MvShape<16, 256, 256, 512, 1> MvV0;     // 16 points, wide blocks
typedef MvShape<16, 256, 256, 512, 2> MvV1;     // 16 points, two blocks per SM (<= 128 registers)
typedef MvShape<8, 256, 512, 512, 1> MvV2;      // 8 points, twice the threads per column
typedef MvShape<8, 256, 256, 256, 2> MvV3;      // 8 points, two blocks per SM
typedef MvShape<8, 64, 64, 64, 4> MvV4;         // 8 points, small blocks (many blocks on small grids)
typedef MvShape<16, 256, 256, 512, 1, 1> MvV5;  // V0 with the pipelined column pass
typedef MvShape<8, 256, 512, 512, 1, 1> MvV6;   // V2 with the pipelined column pass
// 16 points, smaller column blocks, two per SM (each block's barriers hold
// only its own warps, so one block's shared-memory exchanges can overlap the
// other's butterflies).  Measured at L = 2048 (ncu): FP32 column pass 30.3 us
// against 32.6 us for V0 (two columns per 256-thread block); FP64 60.6 us
// against 53.4 us (one column per 128-thread block: its loads use 16 of each
// 32-byte sector of T).
typedef MvShape<16, 256, 128, 256, 2> MvV7;
// V0's transforms with the grouped pipelined column pass (k_cols_convolve_grp):
// each column transform of a block is an independent worker with its own
// staging and named barrier, so one transform's shared-memory exchanges can
// overlap another's butterflies instead of the whole block stepping together.
typedef MvShape<16, 256, 256, 512, 1, 2> MvV8;
// Pipelined forward row pass (k_rows_forward_pipe: persistent workers of 256
// threads, two per block, each staging its next row's x and contrast with
// cp.async while it transforms the current row), 8 points per thread; its
// column pass is V6's.
typedef MvShape<8, 512, 512, 512, 1, 3> MvV9;
constexpr int MV_VARIANTS = 10;

template <int L, typename SH> struct RowCfg {
    typedef Plan<L, SH::E> P;
    static constexpr int TPR = P::TPR;
    static constexpr int RPC = (TPR >= SH::ROWT) ? 1 : SH::ROWT / TPR;
    static constexpr int THREADS = RPC * TPR;
    static constexpr int SMEM_ELEMS = RPC * P::SMEM_ELEMS;
};

template <int L, typename SH, int ESZ> struct ColCfg {
    typedef Plan<L, SH::E> P;
    static constexpr int TPR = P::TPR;
    static constexpr int TARGET = ESZ >= 16 ? SH::COLT64 : SH::COLT32;
    static constexpr int CPB0 = (TPR >= TARGET) ? 1 : TARGET / TPR;
    static constexpr int CPB = CPB0 > L ? L : CPB0;
    static constexpr int THREADS = CPB * TPR;
    // columns interleaved element by element: element i of column c at sm[pad(i) * CPB + c]
    static constexpr int SMEM_ELEMS = P::SMEM_ELEMS * CPB;
};

// ---------------------------------------------------------------- pass 1
template <typename C, int L, typename SH>
__global__ void __launch_bounds__(RowCfg<L, SH>::THREADS, SH::MINB)
k_rows_forward(VecSel xs, const double *__restrict__ xscale, const typename real_of<C>::type *__restrict__ cdiag,
               C *__restrict__ T, const C *__restrict__ tw, int N, const DevState *st, int gate, SysSel sy) {
    typedef typename real_of<C>::type R;
    typedef Plan<L, SH::E> P;
    constexpr int E = P::E, TPR = P::TPR;
    st = sys_move_bytes(st, sy.ws);
    if (gated(st, gate)) return;
    xscale = sys_move_bytes(xscale, sy.ws);
    if (cdiag) cdiag += (long long)blockIdx.y * sy.c;
    T += (long long)blockIdx.y * sy.T;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lr = threadIdx.x / TPR, t = threadIdx.x % TPR;
    C *sm = reinterpret_cast<C *>(smraw) + lr * P::SMEM_ELEMS;
    const int row = blockIdx.x * RowCfg<L, SH>::RPC + lr;
    const long long ks = sel_index(st, xs);
    const C *x = reinterpret_cast<const C *>(xs.base) + ks * xs.stride + (long long)blockIdx.y * xs.sys;
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
            const R c = cdiag ? cdiag[rb + idx] * s : s;  // cdiag == null: transpose operator
            reg[p] = cscale(v, c);
        }
    }
    fft_run<L, SH::E, false, true>(reg, sm, tw, t);
    if (live) {
        C *out = T + (size_t)row * L;
#pragma unroll
        for (int p = 0; p < E; p++) out[t + p * TPR] = reg[p];
    }
}

// ---------------------------------------------------------------- pass 2
template <typename C, int L, typename SH>
__global__ void __launch_bounds__(ColCfg<L, SH, sizeof(C)>::THREADS, SH::MINB)
k_cols_convolve(C *__restrict__ T, const C *__restrict__ gq, const C *__restrict__ tw, int N, const DevState *st,
                int gate, SysSel sy) {
    typedef Plan<L, SH::E> P;
    typedef ColCfg<L, SH, sizeof(C)> Q;
    constexpr int E = P::E, TPR = P::TPR, CPB = Q::CPB;
    st = sys_move_bytes(st, sy.ws);
    if (gated(st, gate)) return;
    T += (long long)blockIdx.y * sy.T;
    gq += (long long)blockIdx.y * sy.gq;
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
    fft_run<L, SH::E, false, true, CPB>(reg, sm, tw, t);
    const int Lq = L / 2 + 1;
    const int qc = col <= L / 2 ? col : L - col;
#pragma unroll
    for (int p = 0; p < E; p++) {
        const int k1 = t + p * TPR;
        const int qr = k1 <= L / 2 ? k1 : L - k1;
        reg[p] = cmul(reg[p], __ldg(gq + (size_t)qc * Lq + qr));
    }
    fft_run<L, SH::E, true, false, CPB>(reg, sm, tw, t);
#pragma unroll
    for (int p = 0; p < E / 2; p++) {
        const int k = t + p * TPR;
        if (k < N) T[(size_t)k * L + col] = reg[p];
    }
}

// Pass 2, persistent and double-buffered: one block per SM walks the column
// tiles v = blockIdx.x, blockIdx.x + gridDim.x, ...; while it transforms tile
// v, cp.async copies tile v + gridDim.x (rows 0..N-1 of its CPB columns) and
// that tile's CPB quarter-spectrum columns into the other half of a shared
// staging buffer, so the loads of T and of the spectrum leave the critical
// path.  Same arithmetic, in the same order, as k_cols_convolve.
static __device__ __forceinline__ uint32_t cg_smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
template <typename C> static __device__ __forceinline__ void cp_async_elem(C *dst, const C *src) {
    if constexpr (sizeof(C) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(cg_smem_u32(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(cg_smem_u32(dst)), "l"(src) : "memory");
}
// copy of one 4-, 8- or 16-byte value (the type's size)
template <typename T> static __device__ __forceinline__ void cp_async_val(T *dst, const T *src) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8 || sizeof(T) == 16, "cp.async copies 4, 8 or 16 bytes");
    if constexpr (sizeof(T) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(cg_smem_u32(dst)), "l"(src) : "memory");
    else if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(cg_smem_u32(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(cg_smem_u32(dst)), "l"(src) : "memory");
}
static __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND> static __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}

template <int L, typename SH, int ESZ> struct PipeCfg {
    typedef ColCfg<L, SH, ESZ> Q;
    static constexpr int LQ = L / 2 + 1;
    static constexpr int TD = (L / 2) * Q::CPB;       // staged tile: rows < L/2 (N <= L/2)
    static constexpr int GD = ((LQ * Q::CPB + 1) / 2) * 2;  // staged spectrum columns (even count: 16-byte slots)
    static constexpr int SLOT = TD + GD;
    static constexpr int SMEM_ELEMS = Q::SMEM_ELEMS + 2 * SLOT;
};

template <typename C, int L, typename SH>
__global__ void __launch_bounds__(ColCfg<L, SH, sizeof(C)>::THREADS, 1)
k_cols_convolve_pipe(C *__restrict__ T, const C *__restrict__ gq, const C *__restrict__ tw, int N, const DevState *st,
                     int gate, SysSel sy) {
    typedef Plan<L, SH::E> P;
    typedef ColCfg<L, SH, sizeof(C)> Q;
    typedef PipeCfg<L, SH, sizeof(C)> G;
    constexpr int E = P::E, TPR = P::TPR, CPB = Q::CPB, THREADS = Q::THREADS, LQ = G::LQ;
    st = sys_move_bytes(st, sy.ws);
    if (gated(st, gate)) return;
    T += (long long)blockIdx.y * sy.T;
    gq += (long long)blockIdx.y * sy.gq;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sx = reinterpret_cast<C *>(smraw);  // FFT exchange, Q::SMEM_ELEMS
    C *buf = sx + Q::SMEM_ELEMS;           // two staging slots
    const int cl = threadIdx.x % CPB, t = threadIdx.x / CPB;
    C *sm = sx + cl;
    const int ntiles = L / CPB;
    // mirrored tile order, as in k_cols_convolve: neighbouring v share spectrum columns
    auto tile_of = [ntiles](int v) { return (v & 1) ? (ntiles - 1 - (v >> 1)) : (v >> 1); };
    auto issue = [&](int v, int slot) {
        C *td = buf + slot * G::SLOT;
        C *gd = td + G::TD;
        const int col0 = tile_of(v) * CPB;
        for (int e = threadIdx.x; e < N * CPB; e += THREADS)
            cp_async_elem(td + e, T + (size_t)(e / CPB) * L + col0 + (e % CPB));
        for (int e = threadIdx.x; e < LQ * CPB; e += THREADS) {
            const int c = e / LQ, qr = e % LQ;
            const int col = col0 + c;
            const int qc = col <= L / 2 ? col : L - col;
            cp_async_elem(gd + e, gq + (size_t)qc * LQ + qr);
        }
        cp_async_commit();
    };
    // this thread's base twiddles, loaded once for every tile it transforms
    C wb[TwBase<L, SH::E>::COUNT];
    load_tw_base<L, SH::E>(tw, t, wb);
    int v = blockIdx.x;
    if (v < ntiles) issue(v, 0);
    for (int it = 0; v < ntiles; it++, v += gridDim.x) {
        const int slot = it & 1;
        if (v + (int)gridDim.x < ntiles) issue(v + gridDim.x, slot ^ 1);
        else cp_async_commit();  // empty group: the wait below always leaves one group pending
        cp_async_wait<1>();
        __syncthreads();
        const C *td = buf + slot * G::SLOT;
        const C *gd = td + G::TD;
        const int col = tile_of(v) * CPB + cl;
        C reg[E];
#pragma unroll
        for (int p = 0; p < E; p++) {
            const int k = t + p * TPR;
            reg[p] = czero<C>();
            if (p < E / 2 && k < N) reg[p] = td[k * CPB + cl];
        }
        fft_run_wb<L, SH::E, false, true, CPB>(reg, sm, wb, t);
#pragma unroll
        for (int p = 0; p < E; p++) {
            const int k1 = t + p * TPR;
            const int qr = k1 <= L / 2 ? k1 : L - k1;
            reg[p] = cmul(reg[p], gd[cl * LQ + qr]);
        }
        fft_run_wb<L, SH::E, true, false, CPB>(reg, sm, wb, t);
#pragma unroll
        for (int p = 0; p < E / 2; p++) {
            const int k = t + p * TPR;
            if (k < N) T[(size_t)k * L + col] = reg[p];
        }
        __syncthreads();  // this slot is refilled by the next iteration's issue
    }
    cp_async_wait<0>();
}

// Pass 2, grouped: the G = CPB column transforms of a block are independent
// workers.  Worker w = blockIdx.x G + g walks columns w, w + W, ... (W = gridDim.x
// G); it stages its next column (rows 0..N-1 of T) and that column's
// quarter-spectrum column into its own half of a double buffer with cp.async
// while it transforms the current one, and its barriers are the named barrier
// 1 + g of its TPR threads only.  Same arithmetic, in the same order, as
// k_cols_convolve.  Used where TPR is a whole number of warps and G <= 15
// (GrpCfg::OK); otherwise the shape falls back to k_cols_convolve_pipe.
template <int L, typename SH, int ESZ> struct GrpCfg {
    typedef Plan<L, SH::E> P;
    typedef ColCfg<L, SH, ESZ> Q;
    static constexpr int TPR = P::TPR;
    static constexpr int G = Q::CPB;
    static constexpr int THREADS = Q::THREADS;
    static constexpr bool OK = (TPR % 32 == 0) && G <= 15;
    static constexpr int NT = G > 1 ? TPR : 0;  // one group: block barrier
    static constexpr int LQ = L / 2 + 1;
    static constexpr int TD = L / 2;               // staged column: rows < L/2 (N <= L/2)
    static constexpr int GD = ((LQ + 1) / 2) * 2;  // staged spectrum column (even count)
    static constexpr int SLOT = TD + GD;
    static constexpr int GROUP_ELEMS = P::SMEM_ELEMS + 2 * SLOT;
    static constexpr int SMEM_ELEMS = G * GROUP_ELEMS;
};

template <typename C, int L, typename SH>
__global__ void __launch_bounds__(ColCfg<L, SH, sizeof(C)>::THREADS, 1)
k_cols_convolve_grp(C *__restrict__ T, const C *__restrict__ gq, const C *__restrict__ tw, int N, const DevState *st,
                    int gate, SysSel sy) {
    typedef Plan<L, SH::E> P;
    typedef GrpCfg<L, SH, sizeof(C)> G;
    constexpr int E = P::E, TPR = P::TPR, LQ = G::LQ, NT = G::NT;
    st = sys_move_bytes(st, sy.ws);
    if (gated(st, gate)) return;
    T += (long long)blockIdx.y * sy.T;
    gq += (long long)blockIdx.y * sy.gq;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int g = threadIdx.x / TPR, t = threadIdx.x % TPR;
    const int bar = 1 + g;
    C *sm = reinterpret_cast<C *>(smraw) + g * G::GROUP_ELEMS;  // this worker's FFT exchange
    C *buf = sm + P::SMEM_ELEMS;                                // and its two staging slots
    const int W = gridDim.x * G::G;
    auto issue = [&](int col, int slot) {
        C *td = buf + slot * G::SLOT;
        C *gd = td + G::TD;
        for (int e = t; e < N; e += TPR) cp_async_elem(td + e, T + (size_t)e * L + col);
        const int qc = col <= L / 2 ? col : L - col;
        for (int e = t; e < LQ; e += TPR) cp_async_elem(gd + e, gq + (size_t)qc * LQ + e);
        cp_async_commit();
    };
    C wb[TwBase<L, SH::E>::COUNT];  // base twiddles, loaded once for every column
    load_tw_base<L, SH::E>(tw, t, wb);
    int col = blockIdx.x * G::G + g;
    if (col < L) issue(col, 0);
    for (int it = 0; col < L; it++, col += W) {
        const int slot = it & 1;
        if (col + W < L) issue(col + W, slot ^ 1);
        else cp_async_commit();  // empty group: the wait below always leaves one group pending
        cp_async_wait<1>();
        fft_barrier<NT>(bar);
        const C *td = buf + slot * G::SLOT;
        const C *gd = td + G::TD;
        C reg[E];
#pragma unroll
        for (int p = 0; p < E; p++) {
            const int k = t + p * TPR;
            reg[p] = czero<C>();
            if (p < E / 2 && k < N) reg[p] = td[k];
        }
        fft_run_wb<L, SH::E, false, true, 1, NT>(reg, sm, wb, t, bar);
#pragma unroll
        for (int p = 0; p < E; p++) {
            const int k1 = t + p * TPR;
            const int qr = k1 <= L / 2 ? k1 : L - k1;
            reg[p] = cmul(reg[p], gd[qr]);
        }
        fft_run_wb<L, SH::E, true, false, 1, NT>(reg, sm, wb, t, bar);
#pragma unroll
        for (int p = 0; p < E / 2; p++) {
            const int k = t + p * TPR;
            if (k < N) T[(size_t)k * L + col] = reg[p];
        }
        fft_barrier<NT>(bar);  // this slot is refilled by the next iteration's issue
    }
    cp_async_wait<0>();
}

// Pass 1, persistent and double-buffered: the block's G = THREADS / TPR
// transforms are independent workers (named barrier 1 + g, or the block's when
// G = 1).  Worker w = blockIdx.x G + g walks rows w, w + W, ... (W = gridDim.x G)
// and stages its next row of x and of the contrast (contiguous, so every copy
// is coalesced) into its own half of a double buffer with cp.async while it
// transforms the current row; its base twiddles stay in registers.  Same
// arithmetic, in the same order, as k_rows_forward.
template <int L, typename SH, int ESZ> struct RowPipeCfg {
    typedef Plan<L, SH::E> P;
    static constexpr int TPR = P::TPR;
    static constexpr int THREADS = SH::ROWT > TPR ? SH::ROWT : TPR;
    static constexpr int G = THREADS / TPR;
    static constexpr bool OK = (TPR % 32 == 0) && G <= 15 && G * TPR == THREADS;
    static constexpr int NT = G > 1 ? TPR : 0;
    static constexpr int XS = L / 2;  // staged row of x (N <= L/2), elements of the complex type
    static constexpr int CS = L / 2;  // staged row of the contrast, elements of the real type
    static constexpr size_t SLOT_BYTES = (size_t)XS * ESZ + (size_t)CS * (ESZ / 2);
    static constexpr size_t GROUP_BYTES = (size_t)P::SMEM_ELEMS * ESZ + 2 * SLOT_BYTES;
    static constexpr size_t SMEM_BYTES = G * GROUP_BYTES;
};

template <typename C, int L, typename SH>
__global__ void __launch_bounds__(RowPipeCfg<L, SH, sizeof(C)>::THREADS, 1)
k_rows_forward_pipe(VecSel xs, const double *__restrict__ xscale, const typename real_of<C>::type *__restrict__ cdiag,
                    C *__restrict__ T, const C *__restrict__ tw, int N, const DevState *st, int gate, SysSel sy) {
    typedef typename real_of<C>::type R;
    typedef Plan<L, SH::E> P;
    typedef RowPipeCfg<L, SH, sizeof(C)> G;
    constexpr int E = P::E, TPR = P::TPR, NT = G::NT;
    st = sys_move_bytes(st, sy.ws);
    if (gated(st, gate)) return;
    xscale = sys_move_bytes(xscale, sy.ws);
    if (cdiag) cdiag += (long long)blockIdx.y * sy.c;
    T += (long long)blockIdx.y * sy.T;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int g = threadIdx.x / TPR, t = threadIdx.x % TPR;
    const int bar = 1 + g;
    unsigned char *gb = smraw + (size_t)g * G::GROUP_BYTES;
    C *sm = reinterpret_cast<C *>(gb);
    unsigned char *slots = gb + (size_t)P::SMEM_ELEMS * sizeof(C);
    const long long ks = sel_index(st, xs);
    const C *x = reinterpret_cast<const C *>(xs.base) + ks * xs.stride + (long long)blockIdx.y * xs.sys;
    const R s = xscale ? (R)xscale[ks] : (R)1;
    const int W = gridDim.x * G::G;
    auto issue = [&](int row, int slot) {
        C *xd = reinterpret_cast<C *>(slots + slot * G::SLOT_BYTES);
        R *cd = reinterpret_cast<R *>(slots + slot * G::SLOT_BYTES + (size_t)G::XS * sizeof(C));
        const size_t rb = (size_t)row * (size_t)N;
        for (int e = t; e < N; e += TPR) cp_async_val(xd + e, x + rb + e);
        if (cdiag)
            for (int e = t; e < N; e += TPR) cp_async_val(cd + e, cdiag + rb + e);
        cp_async_commit();
    };
    C wb[TwBase<L, SH::E>::COUNT];
    load_tw_base<L, SH::E>(tw, t, wb);
    int row = blockIdx.x * G::G + g;
    if (row < N) issue(row, 0);
    for (int it = 0; row < N; it++, row += W) {
        const int slot = it & 1;
        if (row + W < N) issue(row + W, slot ^ 1);
        else cp_async_commit();  // empty group: the wait below always leaves one group pending
        cp_async_wait<1>();
        fft_barrier<NT>(bar);
        const C *xd = reinterpret_cast<const C *>(slots + slot * G::SLOT_BYTES);
        const R *cd = reinterpret_cast<const R *>(slots + slot * G::SLOT_BYTES + (size_t)G::XS * sizeof(C));
        C reg[E];
#pragma unroll
        for (int p = 0; p < E; p++) {
            const int idx = t + p * TPR;
            reg[p] = czero<C>();
            if (p < E / 2 && idx < N) {
                const R c = cdiag ? cd[idx] * s : s;  // cdiag == null: transpose operator
                reg[p] = cscale(xd[idx], c);
            }
        }
        fft_run_wb<L, SH::E, false, true, 1, NT>(reg, sm, wb, t, bar);
        C *out = T + (size_t)row * L;
#pragma unroll
        for (int p = 0; p < E; p++) out[t + p * TPR] = reg[p];
        fft_barrier<NT>(bar);  // this slot is refilled by the next iteration's issue
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------- pass 3
template <typename C, typename CO, int L, int MODE, typename SH>
__global__ void __launch_bounds__(RowCfg<L, SH>::THREADS, SH::MINB)
k_rows_inverse(const C *__restrict__ T, VecSel xs, const double *__restrict__ xscale, const C *__restrict__ bvec,
               VecSel ys, double *__restrict__ npart, const C *__restrict__ tw, int N, const DevState *st, int gate,
               const typename real_of<C>::type *__restrict__ cout, SysSel sy, double2 shift) {
    typedef typename real_of<C>::type R;
    typedef typename real_of<CO>::type RO;
    typedef Plan<L, SH::E> P;
    constexpr int E = P::E, TPR = P::TPR;
    constexpr int NWARP = (RowCfg<L, SH>::THREADS + 31) / 32;
    st = sys_move_bytes(st, sy.ws);
    if (gated(st, gate)) return;
    T += (long long)blockIdx.y * sy.T;
    xscale = sys_move_bytes(xscale, sy.ws);
    npart = sys_move_bytes(npart, sy.ws);
    if (bvec) bvec += (long long)blockIdx.y * sy.b;
    if (cout) cout += (long long)blockIdx.y * sy.c;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double wsum[NWARP];
    const int lr = threadIdx.x / TPR, t = threadIdx.x % TPR;
    C *sm = reinterpret_cast<C *>(smraw) + lr * P::SMEM_ELEMS;
    const int row = blockIdx.x * RowCfg<L, SH>::RPC + lr;
    const bool live = row < N;
    C reg[E];
    const long long kx = sel_index(st, xs);
    const long long ky = sel_index(st, ys);
    const C *x = reinterpret_cast<const C *>(xs.base) + kx * xs.stride + (long long)blockIdx.y * xs.sys;
    CO *y = reinterpret_cast<CO *>(ys.base) + ky * ys.stride + (long long)blockIdx.y * ys.sys;
    const R s = xscale ? (R)xscale[kx] : (R)1;
    const size_t rb = (size_t)row * (size_t)N;
    // the epilogue's operands x (and b) are loaded before the transform so that
    // their latency overlaps its arithmetic
    C xv[E / 2], bv[E / 2];
#pragma unroll
    for (int p = 0; p < E / 2; p++) {
        const int idx = t + p * TPR;
        const bool ok = live && idx < N;
        xv[p] = ok ? x[rb + idx] : czero<C>();
        bv[p] = (MODE != 0 && ok) ? bvec[rb + idx] : czero<C>();
    }
    if (live) {
        const C *in = T + (size_t)row * L;
#pragma unroll
        for (int p = 0; p < E; p++) reg[p] = in[t + p * TPR];
    } else {
#pragma unroll
        for (int p = 0; p < E; p++) reg[p] = czero<C>();
    }
    fft_run<L, SH::E, true, false>(reg, sm, tw, t);
    double acc = 0.0;
    if (live) {
#pragma unroll
        for (int p = 0; p < E / 2; p++) {
            const int idx = t + p * TPR;
            if (idx < N) {
                if (cout) reg[p] = cscale(reg[p], cout[rb + idx]);  // transpose: contrast after G
                C o;
                if (MODE == 0) {
                    // (A - shift) applied to s x: s (1 - shift) x - G c s x
                    o = csub(cmul(xv[p], mk<C>((R)(s * (1.0 - shift.x)), (R)(-s * shift.y))), reg[p]);
                } else {
                    o = cadd(csub(bv[p], xv[p]), reg[p]);
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
            for (int w = 0; w < NWARP; w++) tot += wsum[w];
            npart[blockIdx.x] = tot;
        }
    }
}

// Pass 3 of one matvec fused with pass 1 of the next, for chains y_{i+1} =
// (A - shift) y_i (the s-step Newton basis): per row, the inverse transform of
// T, the crop and y_{i+1} = (1 - shift) y_i - G c y_i stored as in
// k_rows_inverse (MODE 0, no scaling, no contrast at the crop), then c y_{i+1}
// zero-padded and transformed forward and stored back into the same row of T
// as k_rows_forward would.  The cropped outputs y_{i+1}[t + p TPR] (p < E/2) are
// already in the forward transform's input layout, so y_{i+1} is not read back
// from HBM.  Each block owns its rows of T, which it reads before it writes.
template <typename C, int L, typename SH>
__global__ void __launch_bounds__(RowCfg<L, SH>::THREADS, SH::MINB)
k_rows_inv_fwd(C *__restrict__ T, VecSel xs, VecSel ys, const typename real_of<C>::type *__restrict__ cdiag,
               const C *__restrict__ tw, int N, const DevState *st, int gate, SysSel sy, double2 shift) {
    typedef typename real_of<C>::type R;
    typedef Plan<L, SH::E> P;
    constexpr int E = P::E, TPR = P::TPR;
    st = sys_move_bytes(st, sy.ws);
    if (gated(st, gate)) return;
    T += (long long)blockIdx.y * sy.T;
    cdiag += (long long)blockIdx.y * sy.c;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lr = threadIdx.x / TPR, t = threadIdx.x % TPR;
    C *sm = reinterpret_cast<C *>(smraw) + lr * P::SMEM_ELEMS;
    const int row = blockIdx.x * RowCfg<L, SH>::RPC + lr;
    const bool live = row < N;
    C reg[E];
    const long long kx = sel_index(st, xs);
    const long long ky = sel_index(st, ys);
    const C *x = reinterpret_cast<const C *>(xs.base) + kx * xs.stride + (long long)blockIdx.y * xs.sys;
    C *y = reinterpret_cast<C *>(ys.base) + ky * ys.stride + (long long)blockIdx.y * ys.sys;
    const size_t rb = (size_t)row * (size_t)N;
    C xv[E / 2];
    R cv[E / 2];
#pragma unroll
    for (int p = 0; p < E / 2; p++) {
        const int idx = t + p * TPR;
        const bool ok = live && idx < N;
        xv[p] = ok ? x[rb + idx] : czero<C>();
        cv[p] = ok ? cdiag[rb + idx] : (R)0;
    }
    C *trow = T + (size_t)row * L;
    if (live) {
#pragma unroll
        for (int p = 0; p < E; p++) reg[p] = trow[t + p * TPR];
    } else {
#pragma unroll
        for (int p = 0; p < E; p++) reg[p] = czero<C>();
    }
    fft_run<L, SH::E, true, false>(reg, sm, tw, t);
    const C sc = mk<C>((R)(1.0 - shift.x), (R)(-shift.y));
#pragma unroll
    for (int p = 0; p < E / 2; p++) {
        const int idx = t + p * TPR;
        C o = czero<C>();
        if (live && idx < N) {
            o = csub(cmul(xv[p], sc), reg[p]);
            y[rb + idx] = o;
        }
        reg[p] = cscale(o, cv[p]);
    }
#pragma unroll
    for (int p = E / 2; p < E; p++) reg[p] = czero<C>();
    fft_run<L, SH::E, false, true>(reg, sm, tw, t);
    if (live) {
#pragma unroll
        for (int p = 0; p < E; p++) trow[t + p * TPR] = reg[p];
    }
}

// ------------------------------------------------- full transforms (setup)
template <int L>
__global__ void __launch_bounds__(RowCfg<L, MvV0>::THREADS)
k_rows_fft_full(double2 *__restrict__ A, const double2 *__restrict__ tw) {
    typedef Plan<L, 16> P;
    constexpr int E = P::E, TPR = P::TPR;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lr = threadIdx.x / TPR, t = threadIdx.x % TPR;
    double2 *sm = reinterpret_cast<double2 *>(smraw) + lr * P::SMEM_ELEMS;
    const int row = blockIdx.x * RowCfg<L, MvV0>::RPC + lr;
    const bool live = row < L;
    double2 reg[E];
#pragma unroll
    for (int p = 0; p < E; p++) reg[p] = live ? A[(size_t)row * L + t + p * TPR] : czero<double2>();
    fft_run<L, 16, false, false>(reg, sm, tw, t);
    if (live) {
#pragma unroll
        for (int p = 0; p < E; p++) A[(size_t)row * L + t + p * TPR] = reg[p];
    }
}

template <int L>
__global__ void __launch_bounds__(ColCfg<L, MvV0, 16>::THREADS)
k_cols_fft_full(double2 *__restrict__ A, const double2 *__restrict__ tw) {
    typedef Plan<L, 16> P;
    typedef ColCfg<L, MvV0, 16> Q;
    constexpr int E = P::E, TPR = P::TPR, CPB = Q::CPB;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int cl = threadIdx.x % CPB, t = threadIdx.x / CPB;
    double2 *sm = reinterpret_cast<double2 *>(smraw) + cl;
    const int col = blockIdx.x * CPB + cl;
    double2 reg[E];
#pragma unroll
    for (int p = 0; p < E; p++) reg[p] = A[(size_t)(t + p * TPR) * L + col];
    fft_run<L, 16, false, false, CPB>(reg, sm, tw, t);
#pragma unroll
    for (int p = 0; p < E; p++) A[(size_t)(t + p * TPR) * L + col] = reg[p];
}

// ---------------------------------------------------------------- launchers
template <typename K> static int set_smem(K kern, size_t bytes) { return smem_optin(kern, bytes); }

// The three passes for one launch shape SH and one embedding size L.
// The row passes do not depend on the column fields (COLT64, COLT32, PIPE):
// shapes that differ only in them share one row-pass instantiation.
template <typename SH> using RowShape = MvShape<SH::E, SH::ROWT, 0, 0, SH::MINB, SH::PIPE == 3 ? 3 : 0>;

template <typename SH0, int L> struct Passes {
    typedef RowShape<SH0> SH;  // row passes
    typedef SH0 CS;            // column pass
    static int fwd(int prec, const MatvecArgs &a, VecSel x, const double *xs, const DevState *st, int gate,
                   cudaStream_t s) {
        typedef RowCfg<L, SH> Q;
        const int grid = (a.N + Q::RPC - 1) / Q::RPC;
        if constexpr (SH::PIPE == 3 && RowPipeCfg<L, SH, 16>::OK) {
            typedef RowPipeCfg<L, SH, 16> G64;
            typedef RowPipeCfg<L, SH, 8> G32;
            const int nblk = (a.N + G64::G - 1) / G64::G;
            const int pg = nblk < a.sms ? nblk : a.sms;
            if (prec == 0) {
                auto kern = k_rows_forward_pipe<double2, L, SH>;
                int e = set_smem(kern, G64::SMEM_BYTES);
                if (e) return e;
                kern<<<dim3(pg, a.nsys), G64::THREADS, G64::SMEM_BYTES, s>>>(
                    x, xs, a.transpose ? nullptr : (const double *)a.cdiag, (double2 *)a.T, (const double2 *)a.tw, a.N,
                    st, gate, sys_sel(a));
            } else {
                auto kern = k_rows_forward_pipe<float2, L, SH>;
                int e = set_smem(kern, G32::SMEM_BYTES);
                if (e) return e;
                kern<<<dim3(pg, a.nsys), G32::THREADS, G32::SMEM_BYTES, s>>>(
                    x, xs, a.transpose ? nullptr : (const float *)a.cdiag, (float2 *)a.T, (const float2 *)a.tw, a.N, st,
                    gate, sys_sel(a));
            }
            return (int)cudaGetLastError();
        }
        if (prec == 0) {
            const size_t smem = (size_t)Q::SMEM_ELEMS * sizeof(double2);
            auto kern = k_rows_forward<double2, L, SH>;
            int e = set_smem(kern, smem);
            if (e) return e;
            kern<<<dim3(grid, a.nsys), Q::THREADS, smem, s>>>(x, xs, a.transpose ? nullptr : (const double *)a.cdiag,
                                                              (double2 *)a.T, (const double2 *)a.tw, a.N, st, gate,
                                                              sys_sel(a));
        } else {
            const size_t smem = (size_t)Q::SMEM_ELEMS * sizeof(float2);
            auto kern = k_rows_forward<float2, L, SH>;
            int e = set_smem(kern, smem);
            if (e) return e;
            kern<<<dim3(grid, a.nsys), Q::THREADS, smem, s>>>(x, xs, a.transpose ? nullptr : (const float *)a.cdiag,
                                                              (float2 *)a.T, (const float2 *)a.tw, a.N, st, gate,
                                                              sys_sel(a));
        }
        return (int)cudaGetLastError();
    }

    template <typename C> static int cols_t(const MatvecArgs &a, const DevState *st, int gate, cudaStream_t s) {
        typedef ColCfg<L, CS, sizeof(C)> Q;
        if constexpr (CS::PIPE == 2 && GrpCfg<L, CS, sizeof(C)>::OK) {
            typedef GrpCfg<L, CS, sizeof(C)> G;
            const size_t smem = (size_t)G::SMEM_ELEMS * sizeof(C);
            auto kern = k_cols_convolve_grp<C, L, CS>;
            int e = set_smem(kern, smem);
            if (e) return e;
            const int nblk = (L + G::G - 1) / G::G;
            const int grid = nblk < a.sms ? nblk : a.sms;
            kern<<<dim3(grid, a.nsys), G::THREADS, smem, s>>>((C *)a.T, (const C *)a.gq, (const C *)a.tw, a.N, st, gate,
                                                              sys_sel(a));
            return (int)cudaGetLastError();
        } else if constexpr (CS::PIPE) {
            const size_t smem = (size_t)PipeCfg<L, CS, sizeof(C)>::SMEM_ELEMS * sizeof(C);
            auto kern = k_cols_convolve_pipe<C, L, CS>;
            int e = set_smem(kern, smem);
            if (e) return e;
            const int ntiles = L / Q::CPB;
            const int grid = ntiles < a.sms ? ntiles : a.sms;
            kern<<<dim3(grid, a.nsys), Q::THREADS, smem, s>>>((C *)a.T, (const C *)a.gq, (const C *)a.tw, a.N, st, gate,
                                                              sys_sel(a));
            return (int)cudaGetLastError();
        } else {
            const size_t smem = (size_t)Q::SMEM_ELEMS * sizeof(C);
            auto kern = k_cols_convolve<C, L, CS>;
            int e = set_smem(kern, smem);
            if (e) return e;
            kern<<<dim3(L / Q::CPB, a.nsys), Q::THREADS, smem, s>>>((C *)a.T, (const C *)a.gq, (const C *)a.tw, a.N, st,
                                                                    gate, sys_sel(a));
            return (int)cudaGetLastError();
        }
    }
    static int cols(int prec, const MatvecArgs &a, const DevState *st, int gate, cudaStream_t s) {
        return prec == 0 ? cols_t<double2>(a, st, gate, s) : cols_t<float2>(a, st, gate, s);
    }

    template <typename C, typename CO, int MODE>
    static int inv_t(const MatvecArgs &a, VecSel x, const double *xs, const void *b, VecSel y, double *npart,
                     const DevState *st, int gate, cudaStream_t s, double2 shift) {
        typedef RowCfg<L, SH> Q;
        const size_t smem = (size_t)Q::SMEM_ELEMS * sizeof(C);
        auto kern = k_rows_inverse<C, CO, L, MODE, SH>;
        int e = set_smem(kern, smem);
        if (e) return e;
        const int grid = (a.N + Q::RPC - 1) / Q::RPC;
        typedef typename real_of<C>::type R;
        kern<<<dim3(grid, a.nsys), Q::THREADS, smem, s>>>((const C *)a.T, x, xs, (const C *)b, y, npart,
                                                            (const C *)a.tw, a.N, st, gate,
                                                            a.transpose ? (const R *)a.cdiag : nullptr, sys_sel(a),
                                                            shift);
        return (int)cudaGetLastError();
    }
    static int inv(int prec, int mode, int out_prec, const MatvecArgs &a, VecSel x, const double *xs, const void *b,
                   VecSel y, double *npart, const DevState *st, int gate, cudaStream_t s, double2 sh) {
        if (prec == 0) {
            if (mode == 0) return inv_t<double2, double2, 0>(a, x, xs, b, y, npart, st, gate, s, sh);
            return out_prec == 0 ? inv_t<double2, double2, 1>(a, x, xs, b, y, npart, st, gate, s, sh)
                                 : inv_t<double2, float2, 1>(a, x, xs, b, y, npart, st, gate, s, sh);
        }
        if (mode == 0) return inv_t<float2, float2, 0>(a, x, xs, b, y, npart, st, gate, s, sh);
        return inv_t<float2, float2, 1>(a, x, xs, b, y, npart, st, gate, s, sh);
    }
    template <typename C>
    static int inv_fwd_t(const MatvecArgs &a, VecSel x, VecSel y, const DevState *st, int gate, cudaStream_t s,
                         double2 shift) {
        typedef RowCfg<L, SH> Q;
        typedef typename real_of<C>::type R;
        const size_t smem = (size_t)Q::SMEM_ELEMS * sizeof(C);
        auto kern = k_rows_inv_fwd<C, L, SH>;
        int e = set_smem(kern, smem);
        if (e) return e;
        const int grid = (a.N + Q::RPC - 1) / Q::RPC;
        kern<<<dim3(grid, a.nsys), Q::THREADS, smem, s>>>((C *)a.T, x, y, (const R *)a.cdiag, (const C *)a.tw, a.N, st,
                                                            gate, sys_sel(a), shift);
        return (int)cudaGetLastError();
    }
    static int inv_fwd(int prec, const MatvecArgs &a, VecSel x, VecSel y, const DevState *st, int gate,
                       cudaStream_t s, double2 sh) {
        return prec == 0 ? inv_fwd_t<double2>(a, x, y, st, gate, s, sh) : inv_fwd_t<float2>(a, x, y, st, gate, s, sh);
    }
    static int rpc() { return RowCfg<L, SH>::RPC; }
};

// Calls F<Passes<SH, L>>::run(args...) for the shape selected by `variant`
// (L >= 128) or variant 0 (smaller L).
template <template <typename> class F, typename... A> static int dispatch(int variant, int L, A... args) {
    switch (L) {
        case 16: return F<Passes<MvV0, 16>>::run(args...);
        case 32: return F<Passes<MvV0, 32>>::run(args...);
        case 64: return F<Passes<MvV0, 64>>::run(args...);
        default: break;
    }
#define CG_V_CASES(SH)                                            \
    switch (L) {                                                  \
        case 128: return F<Passes<SH, 128>>::run(args...);        \
        case 256: return F<Passes<SH, 256>>::run(args...);        \
        case 512: return F<Passes<SH, 512>>::run(args...);        \
        case 1024: return F<Passes<SH, 1024>>::run(args...);      \
        case 2048: return F<Passes<SH, 2048>>::run(args...);      \
        case 4096: return F<Passes<SH, 4096>>::run(args...);      \
        default: return -1;                                       \
    }
    switch (variant) {
        case 0: CG_V_CASES(MvV0)
        case 1: CG_V_CASES(MvV1)
        case 2: CG_V_CASES(MvV2)
        case 3: CG_V_CASES(MvV3)
        case 4: CG_V_CASES(MvV4)
        case 5: CG_V_CASES(MvV5)
        case 6: CG_V_CASES(MvV6)
        case 7: CG_V_CASES(MvV7)
        case 8: CG_V_CASES(MvV8)
        case 9: CG_V_CASES(MvV9)
        default: return -1;
    }
#undef CG_V_CASES
}

template <typename PS> struct FwdF {
    static int run(int prec, const MatvecArgs *a, VecSel x, const double *xs, const DevState *st, int gate,
                   cudaStream_t s) {
        return PS::fwd(prec, *a, x, xs, st, gate, s);
    }
};
template <typename PS> struct ColsF {
    static int run(int prec, const MatvecArgs *a, const DevState *st, int gate, cudaStream_t s) {
        return PS::cols(prec, *a, st, gate, s);
    }
};
template <typename PS> struct InvF {
    static int run(int prec, int mode, int out_prec, const MatvecArgs *a, VecSel x, const double *xs, const void *b,
                   VecSel y, double *npart, const DevState *st, int gate, cudaStream_t s, double2 sh) {
        return PS::inv(prec, mode, out_prec, *a, x, xs, b, y, npart, st, gate, s, sh);
    }
};
template <typename PS> struct InvFwdF {
    static int run(int prec, const MatvecArgs *a, VecSel x, VecSel y, const DevState *st, int gate, cudaStream_t s,
                   double2 sh) {
        return PS::inv_fwd(prec, *a, x, y, st, gate, s, sh);
    }
};
template <typename PS> struct RpcF {
    static int run() { return PS::rpc(); }
};

int fft_supported(int L) {
    return L == 16 || L == 32 || L == 64 || L == 128 || L == 256 || L == 512 || L == 1024 || L == 2048 || L == 4096;
}

int matvec_variants(int L) { return L >= 128 ? MV_VARIANTS : 1; }

int matvec_variant_persistent(int v) { return v == 5 || v == 6 || v == 8 || v == 9; }

int rows_per_block(int variant, int L) { return dispatch<RpcF>(variant, L); }

int launch_rows_forward(int prec, const MatvecArgs &a, VecSel x, const double *xs, const DevState *st, int gate,
                        cudaStream_t s) {
    return dispatch<FwdF>(a.vfwd, a.L, prec, &a, x, xs, st, gate, s);
}

int launch_cols_convolve(int prec, const MatvecArgs &a, const DevState *st, int gate, cudaStream_t s) {
    return dispatch<ColsF>(a.vcols, a.L, prec, &a, st, gate, s);
}

int launch_rows_inverse(int prec, int mode, int out_prec, const MatvecArgs &a, VecSel x, const double *xs,
                        const void *b, VecSel y, double *npart, const DevState *st, int gate, cudaStream_t s,
                        double2 shift) {
    return dispatch<InvF>(a.vinv, a.L, prec, mode, out_prec, &a, x, xs, b, y, npart, st, gate, s, shift);
}

int launch_rows_inv_fwd(int prec, const MatvecArgs &a, VecSel x, VecSel y, const DevState *st, int gate,
                        cudaStream_t s, double2 shift) {
    if (a.transpose || !a.cdiag) return (int)cudaErrorInvalidValue;  // chains of the plain operator only
    return dispatch<InvFwdF>(a.vinv, a.L, prec, &a, x, y, st, gate, s, shift);
}

template <int L> static int fft2d_full_t(double2 *A, const double2 *tw, cudaStream_t s) {
    typedef RowCfg<L, MvV0> QR;
    typedef ColCfg<L, MvV0, 16> QC;
    size_t smem = (size_t)QR::SMEM_ELEMS * sizeof(double2);
    auto kr = k_rows_fft_full<L>;
    int e = set_smem(kr, smem);
    if (e) return e;
    kr<<<(L + QR::RPC - 1) / QR::RPC, QR::THREADS, smem, s>>>(A, tw);
    e = (int)cudaGetLastError();
    if (e) return e;
    smem = (size_t)QC::SMEM_ELEMS * sizeof(double2);
    auto kc = k_cols_fft_full<L>;
    e = set_smem(kc, smem);
    if (e) return e;
    kc<<<L / QC::CPB, QC::THREADS, smem, s>>>(A, tw);
    return (int)cudaGetLastError();
}

int launch_fft2d_full_fp64(int L, double2 *A, const double2 *tw, cudaStream_t s) {
    switch (L) {
        case 16: return fft2d_full_t<16>(A, tw, s);
        case 32: return fft2d_full_t<32>(A, tw, s);
        case 64: return fft2d_full_t<64>(A, tw, s);
        case 128: return fft2d_full_t<128>(A, tw, s);
        case 256: return fft2d_full_t<256>(A, tw, s);
        case 512: return fft2d_full_t<512>(A, tw, s);
        case 1024: return fft2d_full_t<1024>(A, tw, s);
        case 2048: return fft2d_full_t<2048>(A, tw, s);
        case 4096: return fft2d_full_t<4096>(A, tw, s);
        default: return -1;
    }
}

}  // namespace cg
