// Learned preconditioner: a spectral-convolution network (Fourier neural
// operator) with hand-written inference and training kernels.
//
// The network maps (chi, k0 h, r) on an H x W grid to an estimate of A^{-1} r
// for the GFIEM operator A = I - k0^2 G diag(chi), and is used as the initial
// guess and as a variable right preconditioner in flexible GMRES:
//
//   s     = rms(r)                                   (per sample)
//   f     = [0.1 chi, k0 h, Re r / s, Im r / s]      (4 features per cell)
//   v0    = P f + p                                  (lift to 32 channels)
//   z_l   = W_l v_l + b_l + S_l(v_l),  l = 0..3      (S_l: spectral convolution)
//   v_l+1 = GELU(z_l) for l < 3, v_4 = z_3
//   q     = GELU(Q1 v_4 + bq1)                       (128 hidden)
//   o     = Q2 q + bq2                               (2 outputs)
//   M(r)  = r + s (o_0 + i o_1)
//
// S_l keeps 2*16 row frequencies (k1 = 0..15 and H-16..H-1) and 16 column
// frequencies (k2 = 0..15) of the real 2-D DFT, mixes channels per mode with
// a complex 32 x 32 matrix R_l[k1, k2], and transforms back (the inverse real
// DFT of the truncated spectrum, as numpy.fft.irfft2).  M is positively
// homogeneous (M(a r) = a M(r), a > 0), which the solver's lazily normalised
// basis relies on.
//
// Arithmetic: activations are stored in BF16 ([cells, 32] channel-last rows);
// the channel mixing W_l and the projection Q1 (and their transposes in the
// backward pass) run on the tcgen05 tensor cores (BF16 operands, FP32
// accumulation in TMEM, cg_umma.cuh) with the bias, spectral branch, GELU and
// output stages fused into the GEMM epilogue; the truncated DFTs and the
// per-mode mixing run in FP32 on the CUDA cores; weight gradients are FP32
// reductions with fixed summation order (deterministic); Adam keeps FP32
// master weights.
//
// The standard construction this follows is Li et al., "Fourier Neural
// Operator for Parametric Partial Differential Equations", ICLR 2021.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <random>
#include <vector>

#include "../../include/cugmres.h"
#include "cg_common.cuh"
#include "cg_fno.h"
#include "cg_umma.cuh"

namespace cg {
namespace fno {

constexpr int C = 32;          // channels
constexpr int NIN = 4;         // input features
constexpr int HID = 128;       // projection hidden width
constexpr int M1 = 16;         // row modes per sign
constexpr int M2 = 16;         // column modes
constexpr int K1N = 2 * M1;    // retained row frequencies
constexpr int NJ = M2 * C;     // (k2, c) columns of a spectral slab
constexpr int LAYERS = 4;
constexpr int HCH = 32;        // rows per block of the row-direction transforms
constexpr float CHI_SCALE = 0.1f;

constexpr long long RSZ = (long long)K1N * M2 * C * C * 2;  // floats of one R_l
constexpr long long LSZ = RSZ + C * C + C;
constexpr long long OFF_P = 0, OFF_PB = C * NIN, OFF_L0 = OFF_PB + C;
__host__ __device__ constexpr long long off_r(int l) { return OFF_L0 + l * LSZ; }
__host__ __device__ constexpr long long off_w(int l) { return off_r(l) + RSZ; }
__host__ __device__ constexpr long long off_b(int l) { return off_w(l) + C * C; }
constexpr long long OFF_Q1 = OFF_L0 + LAYERS * LSZ;
constexpr long long OFF_BQ1 = OFF_Q1 + HID * C;
constexpr long long OFF_Q2 = OFF_BQ1 + HID;
constexpr long long OFF_BQ2 = OFF_Q2 + 2 * HID;
constexpr long long NPARAM = OFF_BQ2 + 2;

constexpr int RED_THREADS = 256;
constexpr int WG_TILE = 32;  // cells per shared-memory tile of the weight-gradient reductions

__device__ __forceinline__ bool gated(const int *g) { return g && *(volatile const int *)g; }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
    return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&p);
}
__device__ __forceinline__ float2 unpack2(uint32_t u) {
    __nv_bfloat162 p = *reinterpret_cast<__nv_bfloat162 *>(&u);
    return __bfloat1622float2(p);
}
// 32 BF16 values (64 bytes, 16-byte aligned) <-> FP32
__device__ __forceinline__ void st_bf16x32(__nv_bfloat16 *dst, const float (&v)[32]) {
    uint4 *d = reinterpret_cast<uint4 *>(dst);
#pragma unroll
    for (int q = 0; q < 4; q++)
        d[q] = make_uint4(pack2(v[8 * q], v[8 * q + 1]), pack2(v[8 * q + 2], v[8 * q + 3]),
                          pack2(v[8 * q + 4], v[8 * q + 5]), pack2(v[8 * q + 6], v[8 * q + 7]));
}
__device__ __forceinline__ void ld_bf16x32(const __nv_bfloat16 *src, float (&v)[32]) {
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint4 u = s[q];
        float2 a = unpack2(u.x), b = unpack2(u.y), c = unpack2(u.z), d = unpack2(u.w);
        v[8 * q] = a.x, v[8 * q + 1] = a.y, v[8 * q + 2] = b.x, v[8 * q + 3] = b.y;
        v[8 * q + 4] = c.x, v[8 * q + 5] = c.y, v[8 * q + 6] = d.x, v[8 * q + 7] = d.y;
    }
}

template <typename T> __device__ __forceinline__ float re_of(T v) { return (float)v.x; }
template <typename T> __device__ __forceinline__ float im_of(T v) { return (float)v.y; }

// ------------------------------------------------------------ per-sample statistics
// Partial sums of |r|^2 (and, for training, of |x - r|^2) over blocks of a sample.
template <typename RT>
__global__ void __launch_bounds__(RED_THREADS)
k_norm_part(const RT *__restrict__ r, const cg_c64 *__restrict__ x, long long hw, int nbx, double *part,
            const int *gate) {
    if (gated(gate)) return;
    const int b = blockIdx.y;
    const RT *rb = r + (long long)b * hw;
    const cg_c64 *xb = x ? x + (long long)b * hw : nullptr;
    double a = 0.0, t = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < hw; e += (long long)nbx * blockDim.x) {
        const RT v = rb[e];
        a += (double)v.x * v.x + (double)v.y * v.y;
        if (xb) {
            const double dx = (double)xb[e].re - (double)v.x, dy = (double)xb[e].im - (double)v.y;
            t += dx * dx + dy * dy;
        }
    }
    __shared__ double sa[RED_THREADS / 32], st[RED_THREADS / 32];
    a = warp_sum(a);
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) sa[threadIdx.x >> 5] = a, st[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double A = 0, T = 0;
        for (int i = 0; i < RED_THREADS / 32; i++) A += sa[i], T += st[i];
        part[((long long)b * nbx + blockIdx.x) * 2] = A;
        part[((long long)b * nbx + blockIdx.x) * 2 + 1] = T;
    }
}

// s_b = rms(r_b), inv_s_b = 1 / s_b (1 for a zero sample); for training
// wts_b = 1 / (B * ||(x_b - r_b) / s_b||^2).
__global__ void k_norm_fin(const double *part, int nbx, int B, long long hw, float *s, float *inv_s, float *wts,
                           const int *gate) {
    if (gated(gate)) return;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    double A = 0, T = 0;
    for (int i = 0; i < nbx; i++) A += part[((long long)b * nbx + i) * 2], T += part[((long long)b * nbx + i) * 2 + 1];
    const double rms = sqrt(A / (double)hw);
    s[b] = (float)rms;
    const double is = rms > 0.0 ? 1.0 / rms : 1.0;
    inv_s[b] = (float)is;
    if (wts) {
        const double tn = T * is * is;
        wts[b] = (float)(1.0 / ((double)B * (tn > 1e-30 ? tn : 1e-30)));
    }
}

// Channel-major copy of cell e's 32 channels: vT[line][c][w], line = e / W,
// w = e % W (the operand layout of the tensor-core column DFT).  The lanes of
// a warp hold consecutive cells, so each store of a channel is coalesced.
__device__ __forceinline__ void st_channel_major(__nv_bfloat16 *vT, long long e, int W, const float (&v)[32]) {
    const long long line = e / W;
    const int w = (int)(e - line * W);
    __nv_bfloat16 *d = vT + line * (long long)C * W + w;
#pragma unroll
    for (int c = 0; c < C; c++) d[(long long)c * W] = __float2bfloat16(v[c]);
}

// --------------------------------------------------------------------- lift
template <typename RT>
__global__ void __launch_bounds__(256)
k_lift(const RT *__restrict__ r, const float *__restrict__ chi, const float *__restrict__ k0h,
       const float *__restrict__ inv_s, long long hw, long long cells, const float *__restrict__ prm,
       __nv_bfloat16 *__restrict__ v0, __nv_bfloat16 *__restrict__ vT, int W, const int *gate) {
    if (gated(gate)) return;
    __shared__ float P[C * NIN + C];
    for (int i = threadIdx.x; i < C * NIN + C; i += blockDim.x) P[i] = prm[OFF_P + i];
    __syncthreads();
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cells;
         e += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(e / hw);
        const RT rv = r[e];
        const float is = inv_s[b];
        const float f0 = chi[e] * CHI_SCALE, f1 = k0h[b], f2 = re_of(rv) * is, f3 = im_of(rv) * is;
        float v[32];
#pragma unroll
        for (int c = 0; c < C; c++)
            v[c] = P[C * NIN + c] + P[c * NIN] * f0 + P[c * NIN + 1] * f1 + P[c * NIN + 2] * f2 + P[c * NIN + 3] * f3;
        st_bf16x32(v0 + e * C, v);
        if (vT) st_channel_major(vT, e, W, v);
    }
}

// -------------------------------------------------------- column-direction DFTs
// X[line][k2][c] = sc(k2) sum_w v[line][w][c] e^{-2 pi i w k2 / W},
// sc(0) = s0, sc(k2 > 0) = s1.  One block (512 threads = 16 k2 x 32 c) per
// grid line; the line is staged in shared memory as FP32.
__global__ void __launch_bounds__(512)
k_dft_w_fwd(const __nv_bfloat16 *__restrict__ v, int W, const float2 *__restrict__ tw, float2 *__restrict__ X,
            float s0, float s1, const int *gate) {
    if (gated(gate)) return;
    extern __shared__ float smf[];
    float *line = smf;                              // [W][C]
    float2 *t = reinterpret_cast<float2 *>(smf + (size_t)W * C);  // [W]
    const long long ln = blockIdx.x;
    const uint4 *src = reinterpret_cast<const uint4 *>(v + ln * (long long)W * C);
    for (int q = threadIdx.x; q < W * C / 8; q += blockDim.x) {
        const uint4 u = src[q];
        const float2 a = unpack2(u.x), b = unpack2(u.y), c = unpack2(u.z), d = unpack2(u.w);
        float *o = line + (size_t)q * 8;
        o[0] = a.x, o[1] = a.y, o[2] = b.x, o[3] = b.y, o[4] = c.x, o[5] = c.y, o[6] = d.x, o[7] = d.y;
    }
    for (int m = threadIdx.x; m < W; m += blockDim.x) t[m] = tw[m];
    __syncthreads();
    const int k2 = threadIdx.x >> 5, c = threadIdx.x & 31;
    float re = 0.f, im = 0.f;
    int idx = 0;
    for (int w = 0; w < W; w++) {
        const float x = line[w * C + c];
        const float2 e = t[idx];
        re = fmaf(x, e.x, re);
        im = fmaf(-x, e.y, im);
        idx += k2;
        if (idx >= W) idx -= W;
    }
    const float sc = k2 == 0 ? s0 : s1;
    X[(ln * M2 + k2) * C + c] = make_float2(re * sc, im * sc);
}

// out[line][w][c] = sum_k2 sc(k2) Re(Y[line][k2][c] e^{+2 pi i w k2 / W}).
__global__ void __launch_bounds__(256)
k_dft_w_inv(const float2 *__restrict__ Y, int W, const float2 *__restrict__ tw, float *__restrict__ out, float s0,
            float s1, const int *gate) {
    if (gated(gate)) return;
    extern __shared__ float smf[];
    float2 *y = reinterpret_cast<float2 *>(smf);  // [M2][C]
    float2 *t = y + NJ;                            // [W]
    const long long ln = blockIdx.x;
    for (int q = threadIdx.x; q < NJ; q += blockDim.x) {
        const float2 a = Y[ln * NJ + q];
        const float sc = (q / C) == 0 ? s0 : s1;
        y[q] = make_float2(a.x * sc, a.y * sc);
    }
    for (int m = threadIdx.x; m < W; m += blockDim.x) t[m] = tw[m];
    __syncthreads();
    const int c = threadIdx.x & 31;
    for (int w = threadIdx.x >> 5; w < W; w += blockDim.x >> 5) {
        float acc = 0.f;
        int idx = 0;
#pragma unroll
        for (int k2 = 0; k2 < M2; k2++) {
            const float2 a = y[k2 * C + c], e = t[idx];
            acc = fmaf(a.x, e.x, acc);
            acc = fmaf(-a.y, e.y, acc);
            idx += w;
            if (idx >= W) idx -= W;
        }
        out[(ln * W + w) * C + c] = acc;
    }
}

// ----------------------------------------------------------- row-direction DFTs
// Partial forward transform over the rows of chunk hc:
//   P[b][hc][i][j] = sum_{h in chunk} X[b][h][j] e^{-2 pi i h k1_i / H},
// k1_i = i (i < 16), H - 32 + i (i >= 16).  With q = 0..16 and
// w_q = e^{+2 pi i q h / H}: k1 = q uses conj(w_q), k1 = H - q uses w_q.
__global__ void __launch_bounds__(128)
k_dft_h_fwd(const float2 *__restrict__ X, int H, int HC, const float2 *__restrict__ twh, float2 *__restrict__ P,
            const int *gate) {
    if (gated(gate)) return;
    extern __shared__ float2 tws[];
    for (int m = threadIdx.x; m < H; m += blockDim.x) tws[m] = twh[m];
    __syncthreads();
    const int b = blockIdx.x / HC, hc = blockIdx.x % HC;
    const int j = blockIdx.y * 128 + threadIdx.x;
    float2 acc[K1N];
#pragma unroll
    for (int i = 0; i < K1N; i++) acc[i] = make_float2(0.f, 0.f);
    const int h0 = hc * HCH, h1 = min(H, h0 + HCH);
    for (int h = h0; h < h1; h++) {
        const float2 x = X[((long long)b * H + h) * NJ + j];
        int id = 0;
#pragma unroll
        for (int q = 0; q <= M1; q++) {
            const float2 e = tws[id];
            if (q < M1) {  // x * conj(e)
                acc[q].x += x.x * e.x + x.y * e.y;
                acc[q].y += x.y * e.x - x.x * e.y;
            }
            if (q >= 1) {  // x * e, frequency H - q (slot K1N - q)
                acc[K1N - q].x += x.x * e.x - x.y * e.y;
                acc[K1N - q].y += x.y * e.x + x.x * e.y;
            }
            id += h;
            if (id >= H) id -= H;
        }
    }
    float2 *dst = P + ((long long)(b * HC + hc) * K1N) * NJ + j;
#pragma unroll
    for (int i = 0; i < K1N; i++) dst[(long long)i * NJ] = acc[i];
}

// Y1[b][h][j] = sum_i Y2[b][i][j] e^{+2 pi i h k1_i / H}.
__global__ void __launch_bounds__(128)
k_dft_h_inv(const float2 *__restrict__ Y2, int H, int HC, const float2 *__restrict__ twh, float2 *__restrict__ Y1,
            const int *gate) {
    if (gated(gate)) return;
    extern __shared__ float2 tws[];
    for (int m = threadIdx.x; m < H; m += blockDim.x) tws[m] = twh[m];
    __syncthreads();
    const int b = blockIdx.x / HC, hc = blockIdx.x % HC;
    const int j = blockIdx.y * 128 + threadIdx.x;
    float2 y[K1N];
#pragma unroll
    for (int i = 0; i < K1N; i++) y[i] = Y2[((long long)b * K1N + i) * NJ + j];
    const int h0 = hc * HCH, h1 = min(H, h0 + HCH);
    for (int h = h0; h < h1; h++) {
        float2 acc = make_float2(0.f, 0.f);
        int id = 0;
#pragma unroll
        for (int q = 0; q <= M1; q++) {
            const float2 e = tws[id];
            if (q < M1) {  // y_q * e
                acc.x += y[q].x * e.x - y[q].y * e.y;
                acc.y += y[q].x * e.y + y[q].y * e.x;
            }
            if (q >= 1) {  // y_{32-q} * conj(e)
                const float2 a = y[K1N - q];
                acc.x += a.x * e.x + a.y * e.y;
                acc.y += a.y * e.x - a.x * e.y;
            }
            id += h;
            if (id >= H) id -= H;
        }
        Y1[((long long)b * H + h) * NJ + j] = acc;
    }
}

// --------------------------------------------------------------- mode mixing
// Per retained mode (one block): X2 = sum of the row-transform partials,
// Y2[b][o] = sum_c X2[b][c] R[c][o] (R = R_l[k1, k2], complex 32 x 32).
__global__ void __launch_bounds__(256)
k_mix_fwd(const float2 *__restrict__ P, int B, int HC, const float *__restrict__ prm, int layer, float2 *X2save,
          float2 *__restrict__ Y2, const int *gate) {
    if (gated(gate)) return;
    const int mode = blockIdx.x, i = mode / M2, k2 = mode % M2;
    __shared__ float2 R[C * C];
    __shared__ float2 xs[8][C];
    const float2 *Rg = reinterpret_cast<const float2 *>(prm + off_r(layer)) + (long long)mode * C * C;
    for (int q = threadIdx.x; q < C * C; q += blockDim.x) R[q] = Rg[q];
    const int o = threadIdx.x & 31, bl = threadIdx.x >> 5;
    for (int b0 = 0; b0 < B; b0 += 8) {
        __syncthreads();
        const int b = b0 + bl;
        if (b < B) {
            float2 x = make_float2(0.f, 0.f);
            for (int hc = 0; hc < HC; hc++) {
                const float2 p = P[(((long long)b * HC + hc) * K1N + i) * NJ + k2 * C + o];
                x.x += p.x, x.y += p.y;
            }
            xs[bl][o] = x;
            if (X2save) X2save[((long long)b * K1N + i) * NJ + k2 * C + o] = x;
        }
        __syncthreads();
        if (b < B) {
            float2 y = make_float2(0.f, 0.f);
#pragma unroll 8
            for (int c = 0; c < C; c++) {
                const float2 x = xs[bl][c], r = R[c * C + o];
                y.x += x.x * r.x - x.y * r.y;
                y.y += x.x * r.y + x.y * r.x;
            }
            Y2[((long long)b * K1N + i) * NJ + k2 * C + o] = y;
        }
    }
}

// Adjoint of the mode mixing: dY2 = sum of partials,
//   dX2[b][c] = sum_o dY2[b][o] conj(R[c][o]),  dR[c][o] = sum_b conj(X2[b][c]) dY2[b][o]
// (gradients as d/dRe + i d/dIm).  One block per mode owns dR of the mode.
__global__ void __launch_bounds__(256)
k_mix_bwd(const float2 *__restrict__ P, int B, int HC, const float *__restrict__ prm, int layer,
          const float2 *__restrict__ X2, float2 *__restrict__ dX2, float *__restrict__ grad, const int *gate) {
    if (gated(gate)) return;
    const int mode = blockIdx.x, i = mode / M2, k2 = mode % M2;
    __shared__ float2 R[C * C];
    __shared__ float2 dys[8][C], xs[8][C];
    const float2 *Rg = reinterpret_cast<const float2 *>(prm + off_r(layer)) + (long long)mode * C * C;
    for (int q = threadIdx.x; q < C * C; q += blockDim.x) R[q] = Rg[q];
    const int lane = threadIdx.x & 31, bl = threadIdx.x >> 5;
    float2 dr[4];
#pragma unroll
    for (int q = 0; q < 4; q++) dr[q] = make_float2(0.f, 0.f);
    for (int b0 = 0; b0 < B; b0 += 8) {
        __syncthreads();
        const int b = b0 + bl;
        if (b < B) {
            float2 d = make_float2(0.f, 0.f);
            for (int hc = 0; hc < HC; hc++) {
                const float2 p = P[(((long long)b * HC + hc) * K1N + i) * NJ + k2 * C + lane];
                d.x += p.x, d.y += p.y;
            }
            dys[bl][lane] = d;
            xs[bl][lane] = X2[((long long)b * K1N + i) * NJ + k2 * C + lane];
        } else {
            dys[bl][lane] = make_float2(0.f, 0.f);
            xs[bl][lane] = make_float2(0.f, 0.f);
        }
        __syncthreads();
        if (b < B) {  // dX2[b][c = lane]
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll 8
            for (int o = 0; o < C; o++) {
                const float2 d = dys[bl][o], r = R[lane * C + o];
                acc.x += d.x * r.x + d.y * r.y;
                acc.y += d.y * r.x - d.x * r.y;
            }
            dX2[((long long)b * K1N + i) * NJ + k2 * C + lane] = acc;
        }
        // dR[c][o], c = bl + 8 q, o = lane
        for (int bb = 0; bb < 8; bb++) {
            const float2 d = dys[bb][lane];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float2 x = xs[bb][bl + 8 * q];
                dr[q].x += x.x * d.x + x.y * d.y;
                dr[q].y += x.x * d.y - x.y * d.x;
            }
        }
    }
    float2 *g = reinterpret_cast<float2 *>(grad + off_r(layer)) + (long long)mode * C * C;
#pragma unroll
    for (int q = 0; q < 4; q++) g[(bl + 8 * q) * C + lane] = dr[q];
}

// -------------------------------------------------------------- GEMM epilogues
// Fourier layer, forward: z = acc + b + spectral; v' = GELU(z) (or z).
struct EpiLayer {
    const float *bias;
    const float *spec;
    __nv_bfloat16 *z;
    __nv_bfloat16 *vout;
    __nv_bfloat16 *vT;  // nullable: channel-major copy of vout for the tensor-core column DFT
    int W;
    int act;
    __device__ __forceinline__ void row(long long r, const float (&a)[32], int) {
        float zz[32];
        const float4 *sp = reinterpret_cast<const float4 *>(spec + r * C);
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const float4 s4 = sp[q];
            zz[4 * q] = a[4 * q] + bias[4 * q] + s4.x;
            zz[4 * q + 1] = a[4 * q + 1] + bias[4 * q + 1] + s4.y;
            zz[4 * q + 2] = a[4 * q + 2] + bias[4 * q + 2] + s4.z;
            zz[4 * q + 3] = a[4 * q + 3] + bias[4 * q + 3] + s4.w;
        }
        if (z) st_bf16x32(z + r * C, zz);
        if (act) {
#pragma unroll
            for (int q = 0; q < 32; q++) zz[q] = gelu(zz[q]);
        }
        st_bf16x32(vout + r * C, zz);
        if (vT) st_channel_major(vT, r, W, zz);
    }
    __device__ __forceinline__ void done(long long) {}
};

// Column DFT on the tensor cores for W = 1024 = 32 x 32 (w = 32 w1 + w2): the
// GEMM's A operand is the channel-major activation vT read as rows
// rho = (line C + c) 32 + w1 of the 32 values w2, and B holds the twiddles
// cos / -sin(2 pi w2 k / 1024) of the 16 column modes k (rows 2k, 2k + 1; BF16
// hi and lo parts in two launches, the second adding to the first).  Row rho's
// accumulator is sum_w2 v e^{-2 pi i w2 k / 1024}; the epilogue multiplies it by
// e^{-2 pi i w1 k / 32} and sums over w1, which are the 32 lanes of the warp
// (reduce-scatter: lane j ends with value j = 2k + part), into X[line][k][c].
// Every lane of a warp must take part: M is a multiple of 128 (W = 1024).
struct EpiDftW {
    float *X;            // float2 [lines][M2][C] seen as floats
    const float2 *tw32;  // (cos, sin)(2 pi m / 32)
    int add;
    __device__ __forceinline__ void row(long long rho, const float (&a)[32], int) {
        const int lane = (int)(rho & 31);
        float v[32];
#pragma unroll
        for (int k = 0; k < M2; k++) {
            const float2 e = __ldg(tw32 + ((lane * k) & 31));
            const float re = a[2 * k], im = a[2 * k + 1];
            v[2 * k] = re * e.x + im * e.y;  // (re + i im) (e.x - i e.y)
            v[2 * k + 1] = im * e.x - re * e.y;
        }
#pragma unroll
        for (int sh = 16; sh >= 1; sh >>= 1) {
            const bool up = (lane & sh) != 0;
#pragma unroll
            for (int i = 0; i < sh; i++) {
                const float send = up ? v[i] : v[i + sh];
                const float keep = up ? v[i + sh] : v[i];
                v[i] = keep + __shfl_xor_sync(0xffffffffu, send, sh);
            }
        }
        const long long line = rho >> 10;
        const int c = (int)((rho >> 5) & 31);
        float *dst = X + ((line * M2 + (lane >> 1)) * C + c) * 2 + (lane & 1);
        *dst = add ? *dst + v[0] : v[0];
    }
    __device__ __forceinline__ void done(long long) {}
};

// Inverse column DFT on the tensor cores for W = 1024: rows
// rho = (line 32 + w1) 32 + c of Z (k_zinv: Z[2k] + i Z[2k+1] =
// sc(k) Y[line][k][c] e^{+2 pi i w1 k / 32}, BF16) times B[w2][n] = cos / -sin
// of 2 pi w2 k / 1024 give out[line][32 w1 + w2][c] = sum_k Re(Z_k e^{+2 pi i w2 k / 1024})
// for the 32 w2 of the row; the lanes of a warp are the 32 channels, so each
// output column is one coalesced store.
struct EpiDftWInv {
    float *out;  // FP32 [cells][C]
    __device__ __forceinline__ void row(long long rho, const float (&a)[32], int) {
        const int c = (int)(rho & 31), w1 = (int)((rho >> 5) & 31);
        const long long line = rho >> 10;
        float *dst = out + (line * 1024 + 32 * w1) * C + c;
#pragma unroll
        for (int w2 = 0; w2 < 32; w2++) dst[w2 * C] = a[w2];
    }
    __device__ __forceinline__ void done(long long) {}
};

__global__ void __launch_bounds__(256)
k_zinv(const float2 *__restrict__ Y, long long lines, float s0, float s1, const float2 *__restrict__ tw32,
       __nv_bfloat16 *__restrict__ Z, const int *gate) {
    if (gated(gate)) return;
    for (long long rho = (long long)blockIdx.x * blockDim.x + threadIdx.x; rho < lines * 1024;
         rho += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(rho & 31), w1 = (int)((rho >> 5) & 31);
        const long long line = rho >> 10;
        float z[32];
#pragma unroll
        for (int k = 0; k < M2; k++) {
            const float2 y = Y[(line * M2 + k) * C + c];
            const float sc = k == 0 ? s0 : s1;
            const float2 e = __ldg(tw32 + ((w1 * k) & 31));  // e^{+2 pi i w1 k / 32}
            z[2 * k] = sc * (y.x * e.x - y.y * e.y);
            z[2 * k + 1] = sc * (y.x * e.y + y.y * e.x);
        }
        st_bf16x32(Z + rho * 32, z);
    }
}

// B operands (forward hi rows 0..31, forward lo rows 32..63; inverse rows
// 64..95: B[w2][n], the forward's transpose, BF16) and the 32 outer twiddles.
__global__ void k_tc_dft_twiddles(__nv_bfloat16 *twb, float2 *tw32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 1024) {
        const int n = i >> 5, w2 = i & 31, k = n >> 1;
        double sn, cs;
        sincospi(2.0 * (double)(w2 * k) / 1024.0, &sn, &cs);
        const float v = (n & 1) ? (float)-sn : (float)cs;
        const __nv_bfloat16 hi = __float2bfloat16(v);
        twb[i] = hi;
        twb[1024 + i] = __float2bfloat16(v - __bfloat162float(hi));
        twb[2048 + w2 * 32 + n] = hi;
    }
    if (i < 32) {
        double sn, cs;
        sincospi(2.0 * (double)i / 32.0, &sn, &cs);
        tw32[i] = make_float2((float)cs, (float)sn);
    }
}

// Projection, forward (N = 128 hidden): zq = acc + bq1, q = GELU(zq),
// o = Q2 q + bq2; inference writes z = r + s (o0 + i o1).
template <typename RT> struct EpiProj {
    const float *bq1, *q2, *bq2;
    __nv_bfloat16 *zq;  // [cells][HID] (training)
    float *out2;        // [cells][2] (training)
    const RT *r;
    RT *zout;
    const float *s;
    long long hw;
    float o0, o1;
    __device__ __forceinline__ void row(long long rw, const float (&a)[32], int c0) {
        if (c0 == 0) o0 = o1 = 0.f;
        float zz[32];
#pragma unroll
        for (int j = 0; j < 32; j++) zz[j] = a[j] + bq1[c0 + j];
        if (zq) st_bf16x32(zq + rw * HID + c0, zz);
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const float g = gelu(zz[j]);
            o0 = fmaf(q2[c0 + j], g, o0);
            o1 = fmaf(q2[HID + c0 + j], g, o1);
        }
    }
    __device__ __forceinline__ void done(long long rw) {
        o0 += bq2[0];
        o1 += bq2[1];
        if (out2) {
            out2[2 * rw] = o0;
            out2[2 * rw + 1] = o1;
        }
        if (zout) {
            const float sc = s[rw / hw];
            RT v = r[rw];
            v.x += (decltype(v.x))(sc * o0);
            v.y += (decltype(v.y))(sc * o1);
            zout[rw] = v;
        }
    }
};

// Backward through a channel mixing: dv = acc (+ spectral adjoint); then
// mode 0: store dv (BF16); mode 1: store dv * GELU'(z_prev) (BF16);
// mode 2: store dv (FP32).
struct EpiBwd {
    const float *dspec;
    const __nv_bfloat16 *zprev;
    __nv_bfloat16 *dz;
    float *dv32;
    int mode;
    __device__ __forceinline__ void row(long long r, const float (&a)[32], int) {
        float d[32];
#pragma unroll
        for (int q = 0; q < 32; q++) d[q] = a[q];
        if (dspec) {
            const float4 *sp = reinterpret_cast<const float4 *>(dspec + r * C);
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const float4 s4 = sp[q];
                d[4 * q] += s4.x, d[4 * q + 1] += s4.y, d[4 * q + 2] += s4.z, d[4 * q + 3] += s4.w;
            }
        }
        if (mode == 2) {
            float4 *o = reinterpret_cast<float4 *>(dv32 + r * C);
#pragma unroll
            for (int q = 0; q < 8; q++) o[q] = make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
            return;
        }
        if (mode == 1) {
            float zz[32];
            ld_bf16x32(zprev + r * C, zz);
#pragma unroll
            for (int q = 0; q < 32; q++) d[q] *= gelu_d(zz[q]);
        }
        st_bf16x32(dz + r * C, d);
    }
    __device__ __forceinline__ void done(long long) {}
};

// Plain FP32 store of C = A B^T (the GEMM self-test entry point).
struct EpiStore {
    float *c;
    int n;
    __device__ __forceinline__ void row(long long r, const float (&a)[32], int c0) {
        float4 *o = reinterpret_cast<float4 *>(c + r * n + c0);
#pragma unroll
        for (int q = 0; q < 8; q++) o[q] = make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
    }
    __device__ __forceinline__ void done(long long) {}
};

// ------------------------------------------------------------ loss and output
// Relative squared error per sample: L = sum_b wts_b ||o_b - t_b||^2 with
// t = (x - r) / s; writes dL/do in place of o and block partials of L.
__global__ void __launch_bounds__(RED_THREADS)
k_loss(float *__restrict__ o, const cg_c64 *__restrict__ x, const cg_c64 *__restrict__ r, const float *inv_s,
       const float *wts, long long hw, long long cells, double *part) {
    double l = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cells;
         e += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(e / hw);
        const float is = inv_s[b], w = wts[b];
        const float t0 = (x[e].re - r[e].re) * is, t1 = (x[e].im - r[e].im) * is;
        const float d0 = o[2 * e] - t0, d1 = o[2 * e + 1] - t1;
        l += (double)w * ((double)d0 * d0 + (double)d1 * d1);
        o[2 * e] = 2.f * w * d0;
        o[2 * e + 1] = 2.f * w * d1;
    }
    __shared__ double sl[RED_THREADS / 32];
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0) sl[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int i = 0; i < RED_THREADS / 32; i++) t += sl[i];
        part[blockIdx.x] = t;
    }
}

// Spectral-only last layer (no pointwise path): v = b + spectral (BF16), and
// its backward dz_prev = dspec * GELU'(z_prev).
__global__ void k_spec_bias(const float *__restrict__ spec, const float *__restrict__ bias, __nv_bfloat16 *__restrict__ v,
                            long long cells, const int *gate) {
    if (gated(gate)) return;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cells;
         e += (long long)gridDim.x * blockDim.x) {
        float a[32];
        const float4 *sp = reinterpret_cast<const float4 *>(spec + e * C);
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const float4 s4 = sp[q];
            a[4 * q] = s4.x + bias[4 * q], a[4 * q + 1] = s4.y + bias[4 * q + 1];
            a[4 * q + 2] = s4.z + bias[4 * q + 2], a[4 * q + 3] = s4.w + bias[4 * q + 3];
        }
        st_bf16x32(v + e * C, a);
    }
}
__global__ void k_spec_bwd(const float *__restrict__ dspec, const __nv_bfloat16 *__restrict__ zprev,
                           __nv_bfloat16 *__restrict__ dz, long long cells) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cells;
         e += (long long)gridDim.x * blockDim.x) {
        float d[32], z[32];
        const float4 *sp = reinterpret_cast<const float4 *>(dspec + e * C);
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const float4 s4 = sp[q];
            d[4 * q] = s4.x, d[4 * q + 1] = s4.y, d[4 * q + 2] = s4.z, d[4 * q + 3] = s4.w;
        }
        ld_bf16x32(zprev + e * C, z);
#pragma unroll
        for (int q = 0; q < 32; q++) d[q] *= gelu_d(z[q]);
        st_bf16x32(dz + e * C, d);
    }
}

// dL/do from a caller's dL/dM (M = r + s (o0 + i o1), gradients as d/dRe + i d/dIm).
__global__ void k_dout_from_dm(float *__restrict__ o, const cg_c64 *__restrict__ dm, const float *__restrict__ s,
                               long long hw, long long cells) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cells;
         e += (long long)gridDim.x * blockDim.x) {
        const float sc = s[e / hw];
        o[2 * e] = sc * dm[e].re;
        o[2 * e + 1] = sc * dm[e].im;
    }
}

// Projection backward on the CUDA cores: thread j = hidden unit over a chunk
// of cells: dzq = (Q2^T do) GELU'(zq); partials of dQ2 = sum do GELU(zq)^T and
// dbq2 = sum do.  Partial layout per block: [Q2 (2 x HID), bq2 (2)].
__global__ void __launch_bounds__(HID)
k_proj_bwd(const __nv_bfloat16 *__restrict__ zq, const float *__restrict__ dout, const float *__restrict__ prm,
           long long cells, __nv_bfloat16 *__restrict__ dzq, float *__restrict__ part) {
    const int j = threadIdx.x;
    const float w0 = prm[OFF_Q2 + j], w1 = prm[OFF_Q2 + HID + j];
    const long long per = (cells + gridDim.x - 1) / gridDim.x;
    const long long e0 = (long long)blockIdx.x * per, e1 = min(cells, e0 + per);
    float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
    for (long long e = e0; e < e1; e++) {
        const float z = __bfloat162float(zq[e * HID + j]);
        const float d0 = dout[2 * e], d1 = dout[2 * e + 1];
        const float g = gelu(z);
        a0 = fmaf(d0, g, a0);
        a1 = fmaf(d1, g, a1);
        if (j == 0) b0 += d0, b1 += d1;
        dzq[e * HID + j] = __float2bfloat16_rn((w0 * d0 + w1 * d1) * gelu_d(z));
    }
    float *p = part + (long long)blockIdx.x * (2 * HID + 2);
    p[j] = a0;
    p[HID + j] = a1;
    if (j == 0) p[2 * HID] = b0, p[2 * HID + 1] = b1;
}

// Weight gradient of a channel mixing: dWt[o][i] = sum_cells dY[o] X[i],
// db[o] = sum_cells dY[o]; per-block partials [NO*NI + NO].
template <int NO, int NI>
__global__ void __launch_bounds__(RED_THREADS)
k_wgrad(const __nv_bfloat16 *__restrict__ dY, const __nv_bfloat16 *__restrict__ X, long long cells,
        float *__restrict__ part) {
    constexpr int PER = NO * NI / RED_THREADS;  // outputs per thread (4 or 16), same o, consecutive i
    static_assert(NO * NI % RED_THREADS == 0 && NI % PER == 0, "shape");
    __shared__ float sd[WG_TILE][NO + 1];
    __shared__ float sx[WG_TILE][NI + 4];
    const int t = threadIdx.x;
    const int o = (t * PER) / NI, i0 = (t * PER) % NI;
    float acc[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) acc[q] = 0.f;
    float bacc = 0.f;
    const long long ntile = (cells + WG_TILE - 1) / WG_TILE;
    for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const long long c0 = tile * WG_TILE;
        __syncthreads();
        for (int q = t; q < WG_TILE * NO; q += RED_THREADS) {
            const int rr = q / NO, cc = q % NO;
            sd[rr][cc] = c0 + rr < cells ? __bfloat162float(dY[(c0 + rr) * NO + cc]) : 0.f;
        }
        for (int q = t; q < WG_TILE * NI; q += RED_THREADS) {
            const int rr = q / NI, cc = q % NI;
            sx[rr][cc] = c0 + rr < cells ? __bfloat162float(X[(c0 + rr) * NI + cc]) : 0.f;
        }
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < WG_TILE; rr++) {
            const float d = sd[rr][o];
#pragma unroll
            for (int q = 0; q < PER; q++) acc[q] = fmaf(d, sx[rr][i0 + q], acc[q]);
        }
        if (t < NO)
            for (int rr = 0; rr < WG_TILE; rr++) bacc += sd[rr][t];
    }
    float *p = part + (long long)blockIdx.x * (NO * NI + NO);
#pragma unroll
    for (int q = 0; q < PER; q++) p[o * NI + i0 + q] = acc[q];
    if (t < NO) p[NO * NI + t] = bacc;
}

// Lift backward: dP[c][j] = sum dv0[c] f_j, dpb[c] = sum dv0[c]; thread (c, j).
template <typename RT>
__global__ void __launch_bounds__(C * NIN)
k_lift_bwd(const float *__restrict__ dv0, const RT *__restrict__ r, const float *__restrict__ chi,
           const float *__restrict__ k0h, const float *__restrict__ inv_s, long long hw, long long cells,
           float *__restrict__ part) {
    const int c = threadIdx.x >> 2, jf = threadIdx.x & 3;
    const long long per = (cells + gridDim.x - 1) / gridDim.x;
    const long long e0 = (long long)blockIdx.x * per, e1 = min(cells, e0 + per);
    float a = 0.f, bsum = 0.f;
    for (long long e = e0; e < e1; e++) {
        const int b = (int)(e / hw);
        const float d = dv0[e * C + c];
        float f;
        if (jf == 0) f = chi[e] * CHI_SCALE;
        else if (jf == 1) f = k0h[b];
        else if (jf == 2) f = re_of(r[e]) * inv_s[b];
        else f = im_of(r[e]) * inv_s[b];
        a = fmaf(d, f, a);
        if (jf == 0) bsum += d;
    }
    float *p = part + (long long)blockIdx.x * (C * NIN + C);
    p[c * NIN + jf] = a;
    if (jf == 0) p[C * NIN + c] = bsum;
}

// dst[i] = sum_b part[b][i] (fixed order).
__global__ void k_reduce(const float *__restrict__ part, int nblk, int cnt, float *__restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblk; b++) s += part[(long long)b * cnt + i];
        dst[i] = (float)s;
    }
}
__global__ void k_reduce_d(const double *__restrict__ part, int nblk, double *__restrict__ dst) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nblk; b++) s += part[b];
        *dst = s;
    }
}

// ---------------------------------------------------------------- optimiser
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// BF16 copies of the tensor-core operands: W_l, W_l^T, Q1, Q1^T.
__global__ void k_pack(const float *__restrict__ p, __nv_bfloat16 *__restrict__ wb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < LAYERS * C * C) {
        const int l = t / (C * C), q = t % (C * C), o = q / C, c = q % C;
        const float w = p[off_w(l) + q];
        wb[l * C * C + o * C + c] = __float2bfloat16_rn(w);
        wb[(LAYERS + l) * C * C + c * C + o] = __float2bfloat16_rn(w);
    }
    if (t < HID * C) {
        const int h = t / C, c = t % C;
        const float w = p[OFF_Q1 + t];
        wb[2 * LAYERS * C * C + h * C + c] = __float2bfloat16_rn(w);
        wb[2 * LAYERS * C * C + HID * C + c * HID + h] = __float2bfloat16_rn(w);
    }
}

// --------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mu;

int get_encode() {
    std::lock_guard<std::mutex> lk(g_encode_mu);
    if (g_encode) return 0;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
        q != cudaDriverEntryPointSuccess) {
        cudaGetLastError();
        return -1;
    }
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return 0;
}

// Row-major BF16 [rows, K] as a TMA map with 32 x box_rows boxes and the
// 64-byte swizzle (K * 2 bytes between rows: a multiple of 16; base 16-byte
// aligned; x coordinates used are multiples of 32 elements = 64 bytes).
int make_map(CUtensorMap *m, const void *ptr, long long rows, int K, int box_rows) {
    if (get_encode() || ((uintptr_t)ptr & 15) || K % 32 || rows < 1 || box_rows > 256) return -1;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    cuuint32_t box[2] = {32u, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1u, 1u};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -1;
}

template <int N, int KC, int S> struct GemmShape {
    static constexpr size_t smem = umma::smem_bytes(N, KC, S);
};

template <int N, int KC, int S, class Epi>
int gemm(int sms, const CUtensorMap &ta, const CUtensorMap &tb, long long M, const Epi &e, int *err, const int *gate,
         cudaStream_t s) {
    if (M <= 0) return 0;
    auto kern = umma::k_gemm<N, KC, S, Epi>;
    const size_t smem = GemmShape<N, KC, S>::smem;
    cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce != cudaSuccess) return (int)ce;
    // several CTAs per SM (each holds few TMEM columns) give the row-per-thread
    // epilogues more warps to keep memory traffic in flight
    ce = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                              (int)cudaSharedmemCarveoutMaxShared);
    if (ce != cudaSuccess) return (int)ce;
    // CTAs per SM: as many as the SM's shared memory holds (1 KB reserved per
    // CTA), within the 512 TMEM columns; the occupancy calculator reports one
    // for these kernels.  Measured at 1024^2 (8 layer GEMMs, 2 projections):
    // layer 179 -> 93 us, projection 453 -> 192 us from 1 to 4 CTAs per SM.
    int dev = 0, smem_sm = 0;
    cudaGetDevice(&dev);
    ce = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (ce != cudaSuccess) return (int)ce;
    int per_sm = smem_sm / (int)(smem + 1024);
    static const int force = [] {
        const char *e = getenv("CUGMRES_FNO_GEMM_CTAS");  // diagnostics: CTAs per SM
        return e && *e ? atoi(e) : 0;
    }();
    if (force > 0) per_sm = force;
    per_sm = std::max(1, std::min(per_sm, (int)(512 / umma::tmem_cols(N))));
    const long long tiles = (M + umma::TILE_M - 1) / umma::TILE_M;
    const int grid = (int)std::min<long long>(tiles, (long long)sms * per_sm);
    kern<<<grid, 128, smem, s>>>(ta, tb, M, e, err, gate);
    return (int)cudaGetLastError();
}

}  // namespace fno
}  // namespace cg

using namespace cg;
using namespace cg::fno;

struct cg_fno {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    unsigned long long seed = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // params, grads, Adam moments
    long long step = 0;
    __nv_bfloat16 *wb = nullptr;  // W_l, W_l^T, Q1, Q1^T (BF16)
    CUtensorMap mapW[LAYERS], mapWT[LAYERS], mapQ1, mapQ1T;
    int *err = nullptr;
    // workspace
    long long cap_cells = 0, cap_lines = 0, cap_part = 0, cap_spec = 0;
    long long cap_vt = 0;  // cells of vT (0: not allocated; only W = 1024 grids use it)
    int cap_B = 0;
    unsigned char *ws = nullptr;
    __nv_bfloat16 *act[LAYERS + 1] = {}, *zpre[LAYERS - 1] = {}, *zq = nullptr, *dz[2] = {}, *dzq = nullptr;
    float *spec = nullptr, *out2 = nullptr, *part = nullptr;
    float2 *X1 = nullptr, *Hp = nullptr, *Y2 = nullptr, *X2s[LAYERS] = {};
    float *s = nullptr, *inv_s = nullptr, *wts = nullptr, *k0h = nullptr;
    double *npart = nullptr, *dloss = nullptr;
    // staging of host inputs
    float *chi_in = nullptr;
    cg_c64 *r_in = nullptr, *x_in = nullptr, *z_out = nullptr;
    CUtensorMap mapA[LAYERS + 1], mapDZ[2], mapDZQ;
    long long map_cells = -1;
    // tensor-core column DFT (W = 1024): channel-major activations, B operand, outer twiddles
    __nv_bfloat16 *vT = nullptr, *twb = nullptr;
    float2 *tw32 = nullptr;
    CUtensorMap mapVT, mapTwHi, mapTwLo, mapTwInv;
    // twiddles of the current grid
    int tw_H = 0, tw_W = 0;
    float2 *twh = nullptr, *tww = nullptr;
    float apply_k0h = -1.f;  // k0 h held in k0h[0] for single-vector applications
    bool local_last = true;  // false: the last Fourier layer has no pointwise path (W_3 unused, held at 0)
    int fwd_B = 0, fwd_H = 0, fwd_W = 0;  // batch kept by cugmres_fno_forward_train
    std::mutex mu;
};

namespace {

constexpr int NBX_MAX = 64;

#define FN_CU(x)                              \
    do {                                      \
        cudaError_t e_ = (x);                 \
        if (e_ != cudaSuccess) {              \
            cudaGetLastError();               \
            return CG_ERR_CUDA;               \
        }                                     \
    } while (0)
#define FN_TRY(...)                           \
    do {                                      \
        int s_ = (__VA_ARGS__);               \
        if (s_ != CG_OK) return s_;           \
    } while (0)
#define FN_K(...)                             \
    do {                                      \
        if ((__VA_ARGS__) != 0) {             \
            cudaGetLastError();               \
            return CG_ERR_CUDA;               \
        }                                     \
    } while (0)

bool dev_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

size_t al256(size_t v) { return (v + 255) & ~(size_t)255; }

int reduction_blocks(const cg_fno *f, long long cells) {
    return (int)std::max<long long>(1, std::min<long long>((cells + 255) / 256, 2LL * f->sms));
}

// Workspace for B samples of H x W cells.
int ensure_ws(cg_fno *f, int B, int H, int W) {
    const long long cells = (long long)B * H * W, lines = (long long)B * H;
    const int HC = (H + HCH - 1) / HCH;
    const long long hp = (long long)B * HC * K1N * NJ;
    const int nred = reduction_blocks(f, cells);
    const long long part = std::max<long long>((long long)nred * (HID * C + HID), 2LL * nred + 16);
    // the channel-major copy feeds the tensor-core column DFT, which only W = 1024 grids run
    const long long vt = W == 1024 ? cells : 0;
    if (cells <= f->cap_cells && lines <= f->cap_lines && B <= f->cap_B && hp <= f->cap_spec && part <= f->cap_part &&
        vt <= f->cap_vt)
        return CG_OK;
    const long long nc = std::max(cells, f->cap_cells), nl = std::max(lines, f->cap_lines);
    const long long nvt = std::max(vt, f->cap_vt);
    const int nb = std::max(B, f->cap_B);
    const long long nh = std::max(hp, f->cap_spec), np = std::max(part, f->cap_part);
    size_t off = 0;
    std::vector<std::pair<void **, size_t>> plan;
    auto add = [&](void **ptr, size_t bytes) { plan.push_back({ptr, bytes}); };
    for (int l = 0; l <= LAYERS; l++) add((void **)&f->act[l], (size_t)nc * C * 2);
    f->vT = nullptr;
    if (nvt > 0) add((void **)&f->vT, (size_t)nvt * C * 2);
    for (int l = 0; l < LAYERS - 1; l++) add((void **)&f->zpre[l], (size_t)nc * C * 2);
    add((void **)&f->zq, (size_t)nc * HID * 2);
    add((void **)&f->dz[0], (size_t)nc * C * 2);
    add((void **)&f->dz[1], (size_t)nc * C * 2);
    add((void **)&f->dzq, (size_t)nc * HID * 2);
    add((void **)&f->spec, (size_t)nc * C * 4);
    add((void **)&f->out2, (size_t)nc * 2 * 4);
    add((void **)&f->X1, (size_t)nl * NJ * 8);
    add((void **)&f->Hp, (size_t)nh * 8);
    add((void **)&f->Y2, (size_t)nb * K1N * NJ * 8);
    for (int l = 0; l < LAYERS; l++) add((void **)&f->X2s[l], (size_t)nb * K1N * NJ * 8);
    add((void **)&f->part, (size_t)np * 4);
    add((void **)&f->s, (size_t)nb * 4);
    add((void **)&f->inv_s, (size_t)nb * 4);
    add((void **)&f->wts, (size_t)nb * 4);
    add((void **)&f->k0h, (size_t)nb * 4);
    add((void **)&f->npart, (size_t)nb * NBX_MAX * 2 * 8);
    add((void **)&f->dloss, 64);
    add((void **)&f->chi_in, (size_t)nc * 4);
    add((void **)&f->r_in, (size_t)nc * 8);
    add((void **)&f->x_in, (size_t)nc * 8);
    add((void **)&f->z_out, (size_t)nc * 8);
    for (auto &pp : plan) off += al256(pp.second);
    if (f->ws) {
        FN_CU(cudaStreamSynchronize(f->stream));
        cudaFree(f->ws);
        f->ws = nullptr;
    }
    unsigned char *base = nullptr;
    if (cudaMalloc(&base, off) != cudaSuccess) {
        cudaGetLastError();
        f->cap_cells = f->cap_lines = f->cap_B = 0;
        f->cap_spec = f->cap_part = f->cap_vt = 0;
        f->vT = nullptr;
        return CG_ERR_OOM;
    }
    f->ws = base;
    off = 0;
    for (auto &pp : plan) {
        *pp.first = base + off;
        off += al256(pp.second);
    }
    f->cap_cells = nc;
    f->cap_lines = nl;
    f->cap_B = nb;
    f->cap_spec = nh;
    f->cap_part = np;
    f->cap_vt = nvt;
    f->map_cells = -1;
    return CG_OK;
}

int ensure_maps(cg_fno *f, long long cells) {
    if (f->map_cells == cells) return CG_OK;
    for (int l = 0; l <= LAYERS; l++)
        if (make_map(&f->mapA[l], f->act[l], cells, C, umma::TILE_M)) return CG_ERR_CUDA;
    for (int q = 0; q < 2; q++)
        if (make_map(&f->mapDZ[q], f->dz[q], cells, C, umma::TILE_M)) return CG_ERR_CUDA;
    if (make_map(&f->mapDZQ, f->dzq, cells, HID, umma::TILE_M)) return CG_ERR_CUDA;
    // rows (line, c, w1) x 32 w2; only where the W = 1024 workspace holds vT for these cells
    if (f->vT && f->cap_vt >= cells && make_map(&f->mapVT, f->vT, cells, C, umma::TILE_M)) return CG_ERR_CUDA;
    f->map_cells = cells;
    return CG_OK;
}

int ensure_twiddles(cg_fno *f, int H, int W) {
    if (f->tw_H == H && f->tw_W == W) return CG_OK;
    if (f->twh) cudaFree(f->twh);
    if (f->tww) cudaFree(f->tww);
    f->twh = f->tww = nullptr;
    f->tw_H = f->tw_W = 0;
    std::vector<float2> th(H), tw(W);
    const double pi = 3.14159265358979323846;
    for (int m = 0; m < H; m++) th[m] = make_float2((float)cos(2 * pi * m / H), (float)sin(2 * pi * m / H));
    for (int m = 0; m < W; m++) tw[m] = make_float2((float)cos(2 * pi * m / W), (float)sin(2 * pi * m / W));
    FN_CU(cudaMalloc(&f->twh, sizeof(float2) * H));
    FN_CU(cudaMalloc(&f->tww, sizeof(float2) * W));
    FN_CU(cudaMemcpy(f->twh, th.data(), sizeof(float2) * H, cudaMemcpyHostToDevice));
    FN_CU(cudaMemcpy(f->tww, tw.data(), sizeof(float2) * W, cudaMemcpyHostToDevice));
    f->tw_H = H;
    f->tw_W = W;
    return CG_OK;
}

// The column DFT runs on the tensor cores for W = 1024 (CUGMRES_FNO_TC_DFT=0: never).
bool tc_dft(const cg_fno *f, int W) {
    static const bool on = [] {
        const char *e = getenv("CUGMRES_FNO_TC_DFT");
        return !(e && e[0] == '0');
    }();
    return on && W == 1024 && f->twb != nullptr && f->vT != nullptr;
}

int ensure_tc_dft(cg_fno *f) {
    if (f->twb) return CG_OK;
    FN_CU(cudaMalloc((void **)&f->twb, sizeof(__nv_bfloat16) * 3072));
    FN_CU(cudaMalloc((void **)&f->tw32, sizeof(float2) * 32));
    k_tc_dft_twiddles<<<4, 256, 0, f->stream>>>(f->twb, f->tw32);
    FN_CU(cudaGetLastError());
    if (make_map(&f->mapTwHi, f->twb, C, C, C) || make_map(&f->mapTwLo, f->twb + 1024, C, C, C) ||
        make_map(&f->mapTwInv, f->twb + 2048, C, C, C)) {
        cudaFree(f->twb);
        cudaFree(f->tw32);
        f->twb = nullptr;
        f->tw32 = nullptr;
        return CG_ERR_CUDA;
    }
    FN_CU(cudaStreamSynchronize(f->stream));
    return CG_OK;
}

int prepare_grid(cg_fno *f, int B, int H, int W) {
    if (H < 2 * M1 || W < 2 * M2 || H > 4096 || W > 1024) return CG_ERR_INVALID;
    FN_TRY(ensure_ws(f, B, H, W));
    FN_TRY(ensure_maps(f, (long long)B * H * W));
    FN_TRY(ensure_twiddles(f, H, W));
    if (W == 1024) FN_TRY(ensure_tc_dft(f));
    return CG_OK;
}

size_t dft_w_fwd_smem(int W) { return (size_t)W * C * 4 + (size_t)W * 8; }
size_t dft_w_inv_smem(int W) { return (size_t)NJ * 8 + (size_t)W * 8; }

int set_smem_attrs(int W, int H) {
    if (cudaFuncSetAttribute(k_dft_w_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dft_w_fwd_smem(W)) ||
        cudaFuncSetAttribute(k_dft_w_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dft_w_inv_smem(W)) ||
        cudaFuncSetAttribute(k_dft_h_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, H * 8) ||
        cudaFuncSetAttribute(k_dft_h_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, H * 8))
        return -1;
    return 0;
}

// Spectral branch S_l(in) into f->spec (FP32 [cells][C]); saves X2 when X2save.
// tc: the column DFT runs on the tensor cores from f->vT, the channel-major copy of `in`.
int spectral_fwd(cg_fno *f, const __nv_bfloat16 *in, int B, int H, int W, int layer, float2 *X2save, const int *gate,
                 cudaStream_t s, bool tc) {
    const long long lines = (long long)B * H;
    const int HC = (H + HCH - 1) / HCH;
    if (tc) {
        EpiDftW e;
        e.X = reinterpret_cast<float *>(f->X1);
        e.tw32 = f->tw32;
        e.add = 0;
        FN_K(gemm<32, 1, 6>(f->sms, f->mapVT, f->mapTwHi, lines * W, e, f->err, gate, s));
        e.add = 1;
        FN_K(gemm<32, 1, 6>(f->sms, f->mapVT, f->mapTwLo, lines * W, e, f->err, gate, s));
    } else {
        k_dft_w_fwd<<<(unsigned)lines, 512, dft_w_fwd_smem(W), s>>>(in, W, f->tww, f->X1, 1.f, 1.f, gate);
    }
    k_dft_h_fwd<<<dim3(B * HC, NJ / 128), 128, H * 8, s>>>(f->X1, H, HC, f->twh, f->Hp, gate);
    k_mix_fwd<<<K1N * M2, 256, 0, s>>>(f->Hp, B, HC, f->p, layer, X2save, f->Y2, gate);
    k_dft_h_inv<<<dim3(B * HC, NJ / 128), 128, H * 8, s>>>(f->Y2, H, HC, f->twh, f->X1, gate);
    const float inv = 1.f / ((float)H * (float)W);
    if (tc) {
        // Z reuses the channel-major buffer (its column DFT has run) and its map
        const int zb = (int)std::min<long long>((lines * 1024 + 255) / 256, 8LL * f->sms);
        k_zinv<<<zb, 256, 0, s>>>(f->X1, lines, inv, 2.f * inv, f->tw32, f->vT, gate);
        FN_K(cudaGetLastError());
        EpiDftWInv e;
        e.out = f->spec;
        FN_K(gemm<32, 1, 6>(f->sms, f->mapVT, f->mapTwInv, lines * W, e, f->err, gate, s));
    } else {
        k_dft_w_inv<<<(unsigned)lines, 256, dft_w_inv_smem(W), s>>>(f->X1, W, f->tww, f->spec, inv, 2.f * inv, gate);
    }
    return (int)cudaGetLastError();
}

// Forward pass over B samples.  RT: type of r (double2 / float2 / cg_c64 as
// float2).  zout (nullable): M(r) in RT.  train: keep what the backward needs.
template <typename RT>
int forward(cg_fno *f, cudaStream_t s, int B, int H, int W, const RT *r, const float *chi, RT *zout, bool train,
            const cg_c64 *x, const int *gate) {
    const long long hw = (long long)H * W, cells = B * hw;
    if (set_smem_attrs(W, H)) return CG_ERR_CUDA;
    const int nbx = (int)std::max<long long>(1, std::min<long long>(NBX_MAX, (hw + 4095) / 4096));
    k_norm_part<RT><<<dim3(nbx, B), RED_THREADS, 0, s>>>(r, train ? x : nullptr, hw, nbx, f->npart, gate);
    k_norm_fin<<<(B + 63) / 64, 64, 0, s>>>(f->npart, nbx, B, hw, f->s, f->inv_s, train ? f->wts : nullptr, gate);
    const int lb = (int)std::min<long long>((cells + 255) / 256, 8LL * f->sms);
    const bool tc = tc_dft(f, W);
    k_lift<RT><<<lb, 256, 0, s>>>(r, chi, f->k0h, f->inv_s, hw, cells, f->p, f->act[0], tc ? f->vT : nullptr, W,
                                  gate);
    FN_K(cudaGetLastError());
    for (int l = 0; l < LAYERS; l++) {
        FN_K(spectral_fwd(f, f->act[l], B, H, W, l, train ? f->X2s[l] : nullptr, gate, s, tc));
        if (l == LAYERS - 1 && !f->local_last) {
            k_spec_bias<<<lb, 256, 0, s>>>(f->spec, f->p + off_b(l), f->act[l + 1], cells, gate);
            FN_K(cudaGetLastError());
            continue;
        }
        EpiLayer e;
        e.bias = f->p + off_b(l);
        e.spec = f->spec;
        e.z = (train && l < LAYERS - 1) ? f->zpre[l] : nullptr;
        e.vout = f->act[l + 1];
        e.vT = (tc && l + 1 < LAYERS) ? f->vT : nullptr;  // the next layer's column DFT reads it
        e.W = W;
        e.act = l < LAYERS - 1 ? 1 : 0;
        FN_K(gemm<32, 1, 6>(f->sms, f->mapA[l], f->mapW[l], cells, e, f->err, gate, s));
    }
    EpiProj<RT> ep;
    ep.bq1 = f->p + OFF_BQ1;
    ep.q2 = f->p + OFF_Q2;
    ep.bq2 = f->p + OFF_BQ2;
    ep.zq = train ? f->zq : nullptr;
    ep.out2 = train ? f->out2 : nullptr;
    ep.r = r;
    ep.zout = zout;
    ep.s = f->s;
    ep.hw = hw;
    ep.o0 = ep.o1 = 0.f;
    FN_K(gemm<HID, 1, 4>(f->sms, f->mapA[LAYERS], f->mapQ1, cells, ep, f->err, gate, s));
    return CG_OK;
}

// Backward pass (after forward(train = true) with targets x): gradients into f->g, loss into f->dloss.
// With x: the loss of cugmres_fno_loss_grad; with dm (x null): dL/dM given by the caller.
int backward(cg_fno *f, cudaStream_t s, int B, int H, int W, const cg_c64 *r, const cg_c64 *x, const float *chi,
             const cg_c64 *dm) {
    const long long hw = (long long)H * W, cells = B * hw, lines = (long long)B * H;
    const int HC = (H + HCH - 1) / HCH;
    const int nred = reduction_blocks(f, cells);
    if (x) {
        double *lpart = reinterpret_cast<double *>(f->part);
        k_loss<<<nred, RED_THREADS, 0, s>>>(f->out2, x, r, f->inv_s, f->wts, hw, cells, lpart);
        k_reduce_d<<<1, 32, 0, s>>>(lpart, nred, f->dloss);
    } else {
        k_dout_from_dm<<<nred, RED_THREADS, 0, s>>>(f->out2, dm, f->s, hw, cells);
    }
    FN_K(cudaGetLastError());
    // projection
    k_proj_bwd<<<nred, HID, 0, s>>>(f->zq, f->out2, f->p, cells, f->dzq, f->part);
    k_reduce<<<2, 256, 0, s>>>(f->part, nred, 2 * HID + 2, f->g + OFF_Q2);
    k_wgrad<HID, C><<<nred, RED_THREADS, 0, s>>>(f->dzq, f->act[LAYERS], cells, f->part);
    k_reduce<<<(HID * C + HID + 255) / 256, 256, 0, s>>>(f->part, nred, HID * C + HID, f->g + OFF_Q1);
    FN_K(cudaGetLastError());
    EpiBwd eb;
    eb.dspec = nullptr;
    eb.zprev = nullptr;
    eb.dz = f->dz[0];
    eb.dv32 = nullptr;
    eb.mode = 0;
    FN_K(gemm<32, 4, 2>(f->sms, f->mapDZQ, f->mapQ1T, cells, eb, f->err, nullptr, s));
    int cur = 0;
    const float inv = 1.f / ((float)H * (float)W);
    for (int l = LAYERS - 1; l >= 0; l--) {
        k_wgrad<C, C><<<nred, RED_THREADS, 0, s>>>(f->dz[cur], f->act[l], cells, f->part);
        k_reduce<<<(C * C + C + 255) / 256, 256, 0, s>>>(f->part, nred, C * C + C, f->g + off_w(l));
        const bool spec_only = l == LAYERS - 1 && !f->local_last;
        if (spec_only) FN_CU(cudaMemsetAsync(f->g + off_w(l), 0, sizeof(float) * C * C, s));
        // spectral adjoint: dY1 = adjoint of the inverse column DFT, then rows, modes, rows, columns
        k_dft_w_fwd<<<(unsigned)lines, 512, dft_w_fwd_smem(W), s>>>(f->dz[cur], W, f->tww, f->X1, inv, 2.f * inv,
                                                                      nullptr);
        k_dft_h_fwd<<<dim3(B * HC, NJ / 128), 128, H * 8, s>>>(f->X1, H, HC, f->twh, f->Hp, nullptr);
        k_mix_bwd<<<K1N * M2, 256, 0, s>>>(f->Hp, B, HC, f->p, l, f->X2s[l], f->Y2, f->g, nullptr);
        k_dft_h_inv<<<dim3(B * HC, NJ / 128), 128, H * 8, s>>>(f->Y2, H, HC, f->twh, f->X1, nullptr);
        k_dft_w_inv<<<(unsigned)lines, 256, dft_w_inv_smem(W), s>>>(f->X1, W, f->tww, f->spec, 1.f, 1.f, nullptr);
        FN_K(cudaGetLastError());
        if (spec_only) {  // dv = dspec only; l - 1 >= 0 has GELU
            k_spec_bwd<<<nred, 256, 0, s>>>(f->spec, f->zpre[l - 1], f->dz[cur ^ 1], cells);
            FN_K(cudaGetLastError());
            cur ^= 1;
            continue;
        }
        EpiBwd e;
        e.dspec = f->spec;
        if (l > 0) {
            e.mode = 1;
            e.zprev = f->zpre[l - 1];
            e.dz = f->dz[cur ^ 1];
            e.dv32 = nullptr;
        } else {
            e.mode = 2;
            e.zprev = nullptr;
            e.dz = nullptr;
            e.dv32 = f->spec;  // in place: each row is read, then written, by one thread
        }
        FN_K(gemm<32, 1, 6>(f->sms, f->mapDZ[cur], f->mapWT[l], cells, e, f->err, nullptr, s));
        cur ^= 1;
    }
    k_lift_bwd<float2><<<nred, C * NIN, 0, s>>>(f->spec, reinterpret_cast<const float2 *>(r), chi, f->k0h, f->inv_s,
                                                hw, cells, f->part);
    k_reduce<<<1, 256, 0, s>>>(f->part, nred, C * NIN + C, f->g + OFF_P);
    FN_K(cudaGetLastError());
    return CG_OK;
}

int pack_weights(cg_fno *f, cudaStream_t s) {
    k_pack<<<(HID * C + 255) / 256, 256, 0, s>>>(f->p, f->wb);
    return cudaGetLastError() == cudaSuccess ? CG_OK : CG_ERR_CUDA;
}

int read_err(cg_fno *f) {
    int e = 0;
    if (cudaMemcpy(&e, f->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    return e ? CG_ERR_CUDA : CG_OK;
}

// Stage a host or device array of `bytes` into dst (device) on the net's stream.
int stage(cg_fno *f, void *dst, const void *src, size_t bytes) {
    if (dev_ptr(src)) {
        FN_CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, f->stream));
    } else {
        FN_CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, f->stream));
    }
    return CG_OK;
}

int stage_inputs(cg_fno *f, int B, int H, int W, const float *chi, const float *k0h, const cg_c64 *r,
                 const cg_c64 *x) {
    const size_t cells = (size_t)B * H * W;
    f->fwd_B = 0;
    FN_TRY(stage(f, f->chi_in, chi, cells * 4));
    FN_TRY(stage(f, f->k0h, k0h, (size_t)B * 4));
    f->apply_k0h = -1.f;
    FN_TRY(stage(f, f->r_in, r, cells * 8));
    if (x) FN_TRY(stage(f, f->x_in, x, cells * 8));
    return CG_OK;
}

}  // namespace

namespace cg {
namespace fno {

int prepare(cg_fno *net, int N, float k0h) {
    if (!net) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(net->mu);
    FN_TRY(prepare_grid(net, 1, N, N));
    FN_CU(cudaMemcpy(net->k0h, &k0h, sizeof(float), cudaMemcpyHostToDevice));
    net->apply_k0h = k0h;
    return CG_OK;
}

int apply(cg_fno *net, cudaStream_t s, int N, int prec, const void *r, const float *chi, float k0h, void *z,
          const int *gate) {
    if (!net || !r || !z || !chi) return CG_ERR_INVALID;
    if (net->cap_cells < (long long)N * N || net->tw_H != N || net->tw_W != N || net->apply_k0h != k0h)
        return CG_ERR_INVALID;  // prepare(net, N, k0h) first
    net->fwd_B = 0;
    FN_TRY(ensure_maps(net, (long long)N * N));
    if (prec == 0)
        return forward<double2>(net, s, 1, N, N, (const double2 *)r, chi, (double2 *)z, false, nullptr, gate);
    return forward<float2>(net, s, 1, N, N, (const float2 *)r, chi, (float2 *)z, false, nullptr, gate);
}

int check_error(cg_fno *net) { return net ? read_err(net) : CG_ERR_INVALID; }

int device_of(const cg_fno *net) { return net ? net->device : -1; }

}  // namespace fno
}  // namespace cg

// ------------------------------------------------------------------- C-ABI
extern "C" int cugmres_fno_create(cg_fno **out, int device, unsigned long long seed) {
    if (!out) return CG_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return device < 0 ? CG_ERR_INVALID : CG_ERR_CUDA;
    }
    FN_CU(cudaSetDevice(device));
    cg_fno *f = new cg_fno();
    f->device = device;
    f->seed = seed;
    cudaDeviceGetAttribute(&f->sms, cudaDevAttrMultiProcessorCount, device);
    const size_t pb = sizeof(float) * NPARAM;
    if (cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&f->p, pb) != cudaSuccess || cudaMalloc(&f->g, pb) != cudaSuccess ||
        cudaMalloc(&f->m, pb) != cudaSuccess || cudaMalloc(&f->v, pb) != cudaSuccess ||
        cudaMalloc(&f->wb, sizeof(__nv_bfloat16) * (2 * LAYERS * C * C + 2 * HID * C)) != cudaSuccess ||
        cudaMalloc(&f->err, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        cugmres_fno_destroy(f);
        return CG_ERR_OOM;
    }
    // initial weights: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) for P, W_l, Q1, Q2
    // (Q2 scaled by 0.1 so that M starts close to the identity); R_l uniform(-1, 1) / (C*C) per component.
    std::vector<float> h(NPARAM, 0.f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> u(-1.f, 1.f);
    for (int i = 0; i < C * NIN; i++) h[OFF_P + i] = u(rng) / sqrtf((float)NIN);
    for (int i = 0; i < C; i++) h[OFF_PB + i] = u(rng) / sqrtf((float)NIN);
    for (int l = 0; l < LAYERS; l++) {
        for (long long i = 0; i < RSZ; i++) h[off_r(l) + i] = u(rng) / (float)(C * C);
        for (int i = 0; i < C * C; i++) h[off_w(l) + i] = u(rng) / sqrtf((float)C);
        for (int i = 0; i < C; i++) h[off_b(l) + i] = u(rng) / sqrtf((float)C);
    }
    for (int i = 0; i < HID * C; i++) h[OFF_Q1 + i] = u(rng) / sqrtf((float)C);
    for (int i = 0; i < HID; i++) h[OFF_BQ1 + i] = u(rng) / sqrtf((float)C);
    for (int i = 0; i < 2 * HID; i++) h[OFF_Q2 + i] = 0.1f * u(rng) / sqrtf((float)HID);
    h[OFF_BQ2] = h[OFF_BQ2 + 1] = 0.f;
    int st = cugmres_fno_set_params(f, h.data());
    if (st != CG_OK) {
        cugmres_fno_destroy(f);
        return st;
    }
    *out = f;
    return CG_OK;
}

extern "C" void cugmres_fno_destroy(cg_fno *f) {
    if (!f) return;
    cudaSetDevice(f->device);
    if (f->stream) cudaStreamSynchronize(f->stream);
    cudaFree(f->p);
    cudaFree(f->g);
    cudaFree(f->m);
    cudaFree(f->v);
    cudaFree(f->wb);
    cudaFree(f->twb);
    cudaFree(f->tw32);
    cudaFree(f->err);
    cudaFree(f->ws);
    cudaFree(f->twh);
    cudaFree(f->tww);
    if (f->stream) cudaStreamDestroy(f->stream);
    cudaGetLastError();
    delete f;
}

extern "C" int cugmres_fno_set_local_last(cg_fno *f, int on) {
    if (!f) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(f->mu);
    f->local_last = on != 0;
    f->fwd_B = 0;
    return CG_OK;
}

extern "C" int cugmres_fno_info(const cg_fno *f, cg_fno_info *info) {
    if (!f || !info) return CG_ERR_INVALID;
    info->layers = LAYERS;
    info->width = C;
    info->modes1 = M1;
    info->modes2 = M2;
    info->hidden = HID;
    info->in_features = NIN;
    info->num_params = NPARAM;
    info->steps = f->step;
    return CG_OK;
}

extern "C" int cugmres_fno_get_params(cg_fno *f, float *params) {
    if (!f || !params) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(f->mu);
    FN_CU(cudaSetDevice(f->device));
    FN_CU(cudaStreamSynchronize(f->stream));
    FN_CU(cudaMemcpy(params, f->p, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    return CG_OK;
}

extern "C" int cugmres_fno_set_params(cg_fno *f, const float *params) {
    if (!f || !params) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(f->mu);
    FN_CU(cudaSetDevice(f->device));
    FN_CU(cudaStreamSynchronize(f->stream));
    FN_CU(cudaMemcpy(f->p, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
    FN_CU(cudaMemset(f->m, 0, sizeof(float) * NPARAM));
    FN_CU(cudaMemset(f->v, 0, sizeof(float) * NPARAM));
    FN_CU(cudaMemset(f->err, 0, sizeof(int)));
    f->step = 0;
    f->fwd_B = 0;
    FN_TRY(pack_weights(f, f->stream));
    for (int l = 0; l < LAYERS; l++) {
        if (make_map(&f->mapW[l], f->wb + l * C * C, C, C, C)) return CG_ERR_CUDA;
        if (make_map(&f->mapWT[l], f->wb + (LAYERS + l) * C * C, C, C, C)) return CG_ERR_CUDA;
    }
    if (make_map(&f->mapQ1, f->wb + 2 * LAYERS * C * C, HID, C, HID)) return CG_ERR_CUDA;
    if (make_map(&f->mapQ1T, f->wb + 2 * LAYERS * C * C + HID * C, C, HID, C)) return CG_ERR_CUDA;
    FN_CU(cudaStreamSynchronize(f->stream));
    return CG_OK;
}

extern "C" int cugmres_fno_forward(cg_fno *f, int B, int H, int W, const float *chi, const float *k0h,
                                   const cg_c64 *r, cg_c64 *z) {
    if (!f || B < 1 || !chi || !k0h || !r || !z) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(f->mu);
    FN_CU(cudaSetDevice(f->device));
    FN_TRY(prepare_grid(f, B, H, W));
    FN_TRY(stage_inputs(f, B, H, W, chi, k0h, r, nullptr));
    const size_t cells = (size_t)B * H * W;
    FN_TRY(forward<float2>(f, f->stream, B, H, W, (const float2 *)f->r_in, f->chi_in, (float2 *)f->z_out, false,
                           nullptr, nullptr));
    const cudaMemcpyKind k = dev_ptr(z) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    FN_CU(cudaMemcpyAsync(z, f->z_out, cells * 8, k, f->stream));
    FN_CU(cudaStreamSynchronize(f->stream));
    return read_err(f);
}

static int loss_grad_impl(cg_fno *f, int B, int H, int W, const float *chi, const float *k0h, const cg_c64 *r,
                          const cg_c64 *x, float *loss) {
    FN_TRY(prepare_grid(f, B, H, W));
    FN_TRY(stage_inputs(f, B, H, W, chi, k0h, r, x));
    FN_TRY(forward<float2>(f, f->stream, B, H, W, (const float2 *)f->r_in, f->chi_in, nullptr, true, f->x_in,
                           nullptr));
    FN_TRY(backward(f, f->stream, B, H, W, f->r_in, f->x_in, f->chi_in, nullptr));
    if (loss) {
        double l = 0.0;
        FN_CU(cudaMemcpyAsync(&l, f->dloss, sizeof(double), cudaMemcpyDeviceToHost, f->stream));
        FN_CU(cudaStreamSynchronize(f->stream));
        *loss = (float)l;
    }
    return CG_OK;
}

extern "C" int cugmres_fno_loss_grad(cg_fno *f, int B, int H, int W, const float *chi, const float *k0h,
                                     const cg_c64 *r, const cg_c64 *x, float *loss, float *grad) {
    if (!f || B < 1 || !chi || !k0h || !r || !x) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(f->mu);
    FN_CU(cudaSetDevice(f->device));
    FN_TRY(loss_grad_impl(f, B, H, W, chi, k0h, r, x, loss));
    if (grad) FN_CU(cudaMemcpyAsync(grad, f->g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, f->stream));
    FN_CU(cudaStreamSynchronize(f->stream));
    return read_err(f);
}

static int adam_step(cg_fno *f, float lr) {
    f->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 / (1.0 - pow((double)b1, (double)f->step)));
    const float c2 = (float)(1.0 / (1.0 - pow((double)b2, (double)f->step)));
    k_adam<<<4 * f->sms, 256, 0, f->stream>>>(f->p, f->g, f->m, f->v, NPARAM, lr, b1, b2, 1e-8f, c1, c2);
    FN_K(cudaGetLastError());
    return pack_weights(f, f->stream);
}

extern "C" int cugmres_fno_train_step(cg_fno *f, int B, int H, int W, const float *chi, const float *k0h,
                                      const cg_c64 *r, const cg_c64 *x, float lr, float *loss) {
    if (!f || B < 1 || !chi || !k0h || !r || !x || !(lr >= 0.f)) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(f->mu);
    FN_CU(cudaSetDevice(f->device));
    FN_TRY(loss_grad_impl(f, B, H, W, chi, k0h, r, x, loss));
    FN_TRY(adam_step(f, lr));
    FN_CU(cudaStreamSynchronize(f->stream));
    return read_err(f);
}

extern "C" int cugmres_fno_forward_train(cg_fno *f, int B, int H, int W, const float *chi, const float *k0h,
                                         const cg_c64 *r, cg_c64 *z) {
    if (!f || B < 1 || !chi || !k0h || !r || !z) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(f->mu);
    FN_CU(cudaSetDevice(f->device));
    FN_TRY(prepare_grid(f, B, H, W));
    FN_TRY(stage_inputs(f, B, H, W, chi, k0h, r, nullptr));
    FN_TRY(forward<float2>(f, f->stream, B, H, W, (const float2 *)f->r_in, f->chi_in, (float2 *)f->z_out, true,
                           nullptr, nullptr));
    const size_t cells = (size_t)B * H * W;
    const cudaMemcpyKind k = dev_ptr(z) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    FN_CU(cudaMemcpyAsync(z, f->z_out, cells * 8, k, f->stream));
    FN_CU(cudaStreamSynchronize(f->stream));
    f->fwd_B = B, f->fwd_H = H, f->fwd_W = W;
    return read_err(f);
}

extern "C" int cugmres_fno_backward(cg_fno *f, const cg_c64 *dm, float *grad, float lr) {
    if (!f || !dm || !(lr >= 0.f)) return CG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(f->mu);
    if (f->fwd_B < 1) return CG_ERR_INVALID;  // needs cugmres_fno_forward_train first
    FN_CU(cudaSetDevice(f->device));
    const int B = f->fwd_B, H = f->fwd_H, W = f->fwd_W;
    const size_t cells = (size_t)B * H * W;
    FN_TRY(stage(f, f->x_in, dm, cells * 8));  // x_in is free in this mode
    FN_TRY(backward(f, f->stream, B, H, W, f->r_in, nullptr, f->chi_in, f->x_in));
    f->fwd_B = 0;
    if (grad) FN_CU(cudaMemcpyAsync(grad, f->g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, f->stream));
    if (lr > 0.f) FN_TRY(adam_step(f, lr));
    FN_CU(cudaStreamSynchronize(f->stream));
    return read_err(f);
}

// C = A B^T on the tensor cores (A: M x K, B: N x K, BF16 row-major; C FP32).
extern "C" int cugmres_gemm_bf16(int device, long long M, int N, int K, const uint16_t *A, const uint16_t *B,
                                 float *Cm) {
    if (M < 1 || !A || !B || !Cm || !((N == 32 || N == 128) && (K == 32 || K == 128))) return CG_ERR_INVALID;
    FN_CU(cudaSetDevice(device));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    void *dA = nullptr, *dB = nullptr, *dC = nullptr;
    int *err = nullptr;
    int st = CG_OK;
    if (cudaMalloc(&dA, (size_t)M * K * 2) || cudaMalloc(&dB, (size_t)N * K * 2) ||
        cudaMalloc(&dC, (size_t)M * N * 4) || cudaMalloc(&err, sizeof(int))) {
        cudaGetLastError();
        st = CG_ERR_OOM;
    }
    CUtensorMap ta, tb;
    if (st == CG_OK && (cudaMemcpy(dA, A, (size_t)M * K * 2, cudaMemcpyHostToDevice) ||
                        cudaMemcpy(dB, B, (size_t)N * K * 2, cudaMemcpyHostToDevice) || cudaMemset(err, 0, 4)))
        st = CG_ERR_CUDA;
    if (st == CG_OK && (make_map(&ta, dA, M, K, umma::TILE_M) || make_map(&tb, dB, N, K, N))) st = CG_ERR_CUDA;
    if (st == CG_OK) {
        EpiStore e;
        e.c = (float *)dC;
        e.n = N;
        int r = 0;
        if (N == 32 && K == 32) r = gemm<32, 1, 6>(sms, ta, tb, M, e, err, nullptr, 0);
        else if (N == 128 && K == 32) r = gemm<128, 1, 4>(sms, ta, tb, M, e, err, nullptr, 0);
        else if (N == 32 && K == 128) r = gemm<32, 4, 2>(sms, ta, tb, M, e, err, nullptr, 0);
        else r = gemm<128, 4, 2>(sms, ta, tb, M, e, err, nullptr, 0);
        if (r || cudaDeviceSynchronize() != cudaSuccess) st = CG_ERR_CUDA;
    }
    int he = 0;
    if (st == CG_OK && (cudaMemcpy(&he, err, 4, cudaMemcpyDeviceToHost) || he)) st = CG_ERR_CUDA;
    if (st == CG_OK && cudaMemcpy(Cm, dC, (size_t)M * N * 4, cudaMemcpyDeviceToHost)) st = CG_ERR_CUDA;
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(err);
    cudaGetLastError();
    return st;
}
