// Arnoldi with classical Gram-Schmidt and delayed reorthogonalisation.
//
// CGS2 reads the basis four times per Arnoldi step (h1 = V^H w, w -= V h1,
// h2 = V^H w, w -= V h2).  Here the second (re)orthogonalisation pass of
// each vector is delayed by one step and merged with the first pass of the
// next one (the "DCGS2" scheme of Swirydowicz, Langou, Ananthan, Yang and
// Thomas, "Low synchronization Gram-Schmidt and GMRES algorithms", Numer.
// Linear Algebra Appl. 28 (2021), and Bielich et al., Parallel Computing 112
// (2022)), so each step reads the basis twice.  Notation of step k
// (q_0..q_{k-1} orthonormal, u_k = A q_{k-1} projected once, not yet
// reorthogonalised nor normalised; slot V[k] holds u_k):
//
//   w = A u_k                                   (matvec into slot V[k+1])
//   one dot pass:  a = Q^H u_k, alpha = u_k^H u_k, c = Q^H w, d = u_k^H w
//   nu = sqrt(alpha - |a|^2),  q_k = (u_k - Q a) / nu
//   column k-1 of H:  H(0:k, k-1) = t_{k-1} + a,  H(k, k-1) = nu
//   delta = (d - a^H c) / nu  (= q_k^H w)
//   u_{k+1} = (w - Q c - q_k delta) / nu        (A q_k projected once)
//   t_k = ([c; delta] - H(0:k, 0:k-1) a) / nu  (first-pass coefficients of A q_k)
//   one axpy pass writes q_k into V[k] and u_{k+1} into V[k+1]; its blocks
//   also evaluate the O(k^2) product H a for t_k (a warp per row of H).
//
// Step 0 uses u_0 = r (the residual the cycle starts from), so nu_0 = ||r||.
// Column k-1 is final only at step k, so the Givens update of the least-
// squares problem runs one step behind and a cycle of m columns makes m+1
// operator applications.  The identities assume Q orthonormal; they were
// checked against plain CGS2 (Q and H agree to 2e-15).
#include <stdlib.h>

#include "cg_common.cuh"
#include "cg_internal.h"

namespace cg {

static constexpr int D2_THREADS = 256;
static constexpr int D2_WARPS = D2_THREADS / 32;
// basis vectors per warp work item (J) and elements per lane per loop trip (U)
// are template parameters of k_dots2; variant table below
static constexpr int AX2_THREADS = 256;
static constexpr int STEP_THREADS = 256;

// Grids are sized to whole waves: SMs x resident blocks per SM of the kernel.
template <typename K> static int waves_grid(K kern, int threads, size_t smem, int sms) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return per_sm * sms;
}

// Two FP32 complex values (re0, im0, re1, im1) moved by one 16-byte access:
// the load unit of the FP32 tile-major passes on vectors of even length, so
// that they issue as few load instructions per byte as the FP64 passes.
template <> struct real_of<float4> { typedef float type; };
template <typename CV> struct scalar_of { typedef CV type; };  // complex scalar of a load unit
template <> struct scalar_of<float4> { typedef float2 type; };
template <> __host__ __device__ __forceinline__ float4 czero<float4>() { return make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ float4 cadd(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 csub(float4 a, float4 b) {
    return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
__device__ __forceinline__ float4 cscale(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 cmul(float2 p, float4 a) {
    return make_float4(p.x * a.x - p.y * a.y, p.x * a.y + p.y * a.x, p.x * a.z - p.y * a.w, p.x * a.w + p.y * a.z);
}
// s0 + i s1 += conj(a) u, s2 + i s3 += conj(a) w over the complex values of a load unit
__device__ __forceinline__ void dacc(double2 a, double2 u, double2 w, double &s0, double &s1, double &s2, double &s3) {
    s0 += a.x * u.x + a.y * u.y;
    s1 += a.x * u.y - a.y * u.x;
    s2 += a.x * w.x + a.y * w.y;
    s3 += a.x * w.y - a.y * w.x;
}
__device__ __forceinline__ void dacc(float2 a, float2 u, float2 w, float &s0, float &s1, float &s2, float &s3) {
    s0 += a.x * u.x + a.y * u.y;
    s1 += a.x * u.y - a.y * u.x;
    s2 += a.x * w.x + a.y * w.y;
    s3 += a.x * w.y - a.y * w.x;
}
__device__ __forceinline__ void dacc(float4 a, float4 u, float4 w, float &s0, float &s1, float &s2, float &s3) {
    s0 += (a.x * u.x + a.y * u.y) + (a.z * u.z + a.w * u.w);
    s1 += (a.x * u.y - a.y * u.x) + (a.z * u.w - a.w * u.z);
    s2 += (a.x * w.x + a.y * w.y) + (a.z * w.z + a.w * w.w);
    s3 += (a.x * w.y - a.y * w.x) + (a.z * w.w - a.w * w.z);
}

static __device__ __forceinline__ int part_ld(const KrylovPtrs &kp) { return dots2_part_ld(kp.mcap); }

static __device__ __forceinline__ bool last_block2(unsigned int *ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
        if (is_last) *ticket = 0u;
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// --------------------------------------------------------------- dots2
// For j = 0..k: D1[j] = <V_j, u_k>, D2[j] = <V_j, w> with u_k = V[k], w = V[k+1].
// Work items: groups of D2_J basis vectors; when there are fewer groups than
// warps, each group's element range is split into S slices.
// Tile-major variant of the two-right-hand-side dot pass: each warp owns
// tiles of 32*U consecutive elements, keeps u and w of its tile in registers
// and streams every basis vector q_j (j = 0..k) over the tile exactly once;
// the four real sums of (q_j^H u, q_j^H w) are reduced across the warp with
// shuffles in FP64 and added to the warp's own shared-memory slots, which the
// block then sums in a fixed order (deterministic).  u and w are read once
// from HBM instead of once per group of basis vectors.  FP32 vectors form
// their products in FP32 over the U elements of a lane (FMA), everything after
// that is FP64.  The basis is processed in chunks of cs = min(mcap + 1,
// D2T_CHUNK) vectors (u and w are re-read once per chunk), so shared memory is
// D2_WARPS * cs * 4 doubles (at most 64 KB) whatever the restart length.
static constexpr int D2T_CHUNK = 256;

// Arrival counter over `count` blocks; the last to arrive resets it and
// sees true (with the other blocks' writes visible).
static __device__ __forceinline__ bool last_of(unsigned int *ticket, unsigned int count) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int t = atomicAdd(ticket, 1u);
        is_last = (t == count - 1);
        if (is_last) *ticket = 0u;
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// Two-level fixed-order sum of the per-block partial rows part[b][0 .. 4 njt)
// into D1, D2: the last block of each group of 16 blocks sums its group's
// rows into gpart[g], the last group sums the group rows.  Replaces one block
// reading every row, which dominated the pass on grids of hundreds of blocks.
constexpr int RGROUP = 16;
static __device__ void dots2_finish(const KrylovPtrs &kp, DevState *st, int njt, int pld) {
    const int nb = gridDim.x, ng = (nb + RGROUP - 1) / RGROUP;
    const int g = blockIdx.x / RGROUP;
    const int gsz = nb - g * RGROUP < RGROUP ? nb - g * RGROUP : RGROUP;
    if (!last_of(&kp.tickets[g], (unsigned int)gsz)) return;
    for (int q = threadIdx.x; q < 4 * njt; q += blockDim.x) {
        double s = 0.0;
        for (int b = g * RGROUP; b < g * RGROUP + gsz; b++) s += __ldcg(kp.part + 4 * (size_t)b * pld + q);
        kp.gpart[4 * (size_t)g * pld + q] = s;
    }
    if (!last_of(&st->counter[3], (unsigned int)ng)) return;
    for (int q = threadIdx.x; q < 4 * njt; q += blockDim.x) {
        double s = 0.0;
        for (int gg = 0; gg < ng; gg++) s += __ldcg(kp.gpart + 4 * (size_t)gg * pld + q);
        double2 *dst = (q & 3) < 2 ? kp.D1 : kp.D2;
        reinterpret_cast<double *>(dst + (q >> 2))[q & 1] = s;
    }
}


// Sum of four values over the warp with a reduce-scatter butterfly: 6
// shuffles instead of 4 x 5.  On return lane 8*q holds the total of a_q
// (q = 0..3); the summation order is fixed (deterministic).
__device__ __forceinline__ double warp_sum4_scatter(double a0, double a1, double a2, double a3, int lane) {
    const bool b4 = lane & 16, b3 = lane & 8;
    const double s0 = b4 ? a0 : a2, s1 = b4 ? a1 : a3;
    const double k0 = (b4 ? a2 : a0) + __shfl_xor_sync(0xffffffffu, s0, 16);
    const double k1 = (b4 ? a3 : a1) + __shfl_xor_sync(0xffffffffu, s1, 16);
    double m = (b3 ? k1 : k0) + __shfl_xor_sync(0xffffffffu, b3 ? k0 : k1, 8);
    m += __shfl_xor_sync(0xffffffffu, m, 4);
    m += __shfl_xor_sync(0xffffffffu, m, 2);
    m += __shfl_xor_sync(0xffffffffu, m, 1);
    return m;
}
template <typename CV, int U>
__global__ void __launch_bounds__(D2_THREADS, 2) k_dots2t(const CV *__restrict__ V, long long n, KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    V = sys_vec(V, kp);
    typedef typename real_of<CV>::type R;
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k;
    const int njt = k + 1;
    const CV *u = V + (long long)k * n;
    const CV *w = V + (long long)(k + 1) * n;
    extern __shared__ double sacc[];  // [D2_WARPS][cs][4]
    const int cs = kp.mcap + 1 < D2T_CHUNK ? kp.mcap + 1 : D2T_CHUNK;  // chunk of basis vectors
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *my = sacc + (size_t)warp * cs * 4;
    const int pld = part_ld(kp);
    const long long TILE = 32LL * U;
    const long long ntile = (n + TILE - 1) / TILE;
    const long long nw = (long long)gridDim.x * D2_WARPS;
    for (int jc = 0; jc < njt; jc += cs) {
        const int nj = njt - jc < cs ? njt - jc : cs;
        const CV *Vc = V + (long long)jc * n;
        for (int q = lane; q < nj * 4; q += 32) my[q] = 0.0;
        __syncwarp();
        for (long long tile = (long long)blockIdx.x * D2_WARPS + warp; tile < ntile; tile += nw) {
            const long long e0 = tile * TILE + lane;
            const bool full = tile * TILE + TILE <= n;
            CV uu[U], ww[U], a[U];
#pragma unroll
            for (int t = 0; t < U; t++) {
                const long long e = e0 + 32 * t;
                const bool ok = full || e < n;
                uu[t] = ok ? u[e] : czero<CV>();
                ww[t] = ok ? w[e] : czero<CV>();
                a[t] = ok ? __ldcs(Vc + e) : czero<CV>();
            }
            for (int j = 0; j < nj; j++) {
                R s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
                for (int t = 0; t < U; t++) dacc(a[t], uu[t], ww[t], s0, s1, s2, s3);
                if (j + 1 < nj) {  // next vector's tile in flight during the reduction
                    const CV *vn = Vc + (long long)(j + 1) * n;
#pragma unroll
                    for (int t = 0; t < U; t++) {
                        const long long e = e0 + 32 * t;
                        a[t] = (full || e < n) ? __ldcs(vn + e) : czero<CV>();
                    }
                }
                const double d = warp_sum4_scatter((double)s0, (double)s1, (double)s2, (double)s3, lane);
                if ((lane & 7) == 0) my[4 * j + (lane >> 3)] += d;
            }
        }
        __syncthreads();
        for (int q = threadIdx.x; q < nj * 4; q += blockDim.x) {
            double t = 0.0;
            for (int wq = 0; wq < D2_WARPS; wq++) t += sacc[(size_t)wq * cs * 4 + q];
            kp.part[4 * ((size_t)blockIdx.x * pld + jc) + q] = t;
        }
        __syncthreads();
    }
    dots2_finish(kp, st, njt, pld);
}

// Split variant of the dot pass for grids with few tiles and many basis
// vectors: a block owns a tile of 32*U elements at a time and its warps share
// the basis (warp w takes q_j with j = w mod D2_WARPS), each warp keeping u and
// w of the tile in registers.  Every coefficient j has one owning warp, so the
// block accumulates it in a single shared-memory slot (chunks of cs vectors)
// without atomics; block partials and the last-block sum as in k_dots2t.
template <typename CV, int U>
__global__ void __launch_bounds__(D2_THREADS) k_dots2s(const CV *__restrict__ V, long long n, KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    V = sys_vec(V, kp);
    typedef typename real_of<CV>::type R;
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k;
    const int njt = k + 1;
    const CV *u = V + (long long)k * n;
    const CV *w = V + (long long)(k + 1) * n;
    extern __shared__ double sacc[];  // [cs][4]
    const int cs = kp.mcap + 1 < D2T_CHUNK ? kp.mcap + 1 : D2T_CHUNK;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pld = part_ld(kp);
    const long long TILE = 32LL * U;
    const long long ntile = (n + TILE - 1) / TILE;
    for (int jc = 0; jc < njt; jc += cs) {
        const int nj = njt - jc < cs ? njt - jc : cs;
        const CV *Vc = V + (long long)jc * n;
        for (int q = threadIdx.x; q < nj * 4; q += blockDim.x) sacc[q] = 0.0;
        __syncthreads();
        for (long long tile = blockIdx.x; tile < ntile && warp < nj; tile += gridDim.x) {
            const long long e0 = tile * TILE + lane;
            const bool full = tile * TILE + TILE <= n;
            CV uu[U], ww[U], a[U];
            const CV *v0 = Vc + (long long)warp * n;
#pragma unroll
            for (int t = 0; t < U; t++) {
                const long long e = e0 + 32 * t;
                const bool ok = full || e < n;
                uu[t] = ok ? u[e] : mk<CV>(0, 0);
                ww[t] = ok ? w[e] : mk<CV>(0, 0);
                a[t] = ok ? __ldcs(v0 + e) : mk<CV>(0, 0);
            }
            for (int j = warp; j < nj; j += D2_WARPS) {
                R s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
                for (int t = 0; t < U; t++) {
                    s0 += a[t].x * uu[t].x + a[t].y * uu[t].y;
                    s1 += a[t].x * uu[t].y - a[t].y * uu[t].x;
                    s2 += a[t].x * ww[t].x + a[t].y * ww[t].y;
                    s3 += a[t].x * ww[t].y - a[t].y * ww[t].x;
                }
                if (j + D2_WARPS < nj) {  // this warp's next vector in flight during the reduction
                    const CV *vn = Vc + (long long)(j + D2_WARPS) * n;
#pragma unroll
                    for (int t = 0; t < U; t++) {
                        const long long e = e0 + 32 * t;
                        a[t] = (full || e < n) ? __ldcs(vn + e) : mk<CV>(0, 0);
                    }
                }
                const double d = warp_sum4_scatter((double)s0, (double)s1, (double)s2, (double)s3, lane);
                if ((lane & 7) == 0) sacc[4 * j + (lane >> 3)] += d;
            }
        }
        __syncthreads();
        for (int q = threadIdx.x; q < nj * 4; q += blockDim.x) kp.part[4 * ((size_t)blockIdx.x * pld + jc) + q] = sacc[q];
        __syncthreads();
    }
    dots2_finish(kp, st, njt, pld);
}

template <typename CV, bool COMP, int D2_J, int U>
__global__ void __launch_bounds__(D2_THREADS) k_dots2(const CV *__restrict__ V, long long n, KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    V = sys_vec(V, kp);
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k;
    const int nj = k + 1;
    const CV *u = V + (long long)k * n;
    const CV *w = V + (long long)(k + 1) * n;
    long long chunk = (n + gridDim.x - 1) / gridDim.x;
    chunk = (chunk + 31) & ~31LL;
    const long long b0 = (long long)blockIdx.x * chunk < n ? (long long)blockIdx.x * chunk : n;
    const long long b1 = b0 + chunk < n ? b0 + chunk : n;
    const int ng = (nj + D2_J - 1) / D2_J;
    const int pld = part_ld(kp);
    // split each group's element range into S slices so that the items fill
    // whole rounds of the block's warps (S * nj partials must fit pld)
    int S = 1;
    {
        double best = -1.0;
        for (int cand = 1; cand <= 8; cand++) {
            if (cand * nj > pld) break;
            const int itc = ng * cand;
            const int rounds = (itc + D2_WARPS - 1) / D2_WARPS;
            const double eff = (double)itc / (double)(rounds * D2_WARPS) - 0.02 * cand;
            if (eff > best) {
                best = eff;
                S = cand;
            }
        }
    }
    const int items = ng * S;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int it = warp; it < items; it += D2_WARPS) {
        const int grp = it / S, sl = it % S;
        const int j0 = grp * D2_J;
        const int jn = nj - j0 < D2_J ? nj - j0 : D2_J;
        long long sc = (b1 - b0 + S - 1) / S;
        sc = (sc + 31) & ~31LL;
        const long long e0 = b0 + sl * sc < b1 ? b0 + sl * sc : b1;
        const long long e1 = e0 + sc < b1 ? e0 + sc : b1;
        const CV *vj[D2_J];
#pragma unroll
        for (int q = 0; q < D2_J; q++) vj[q] = V + (long long)(j0 + (q < jn ? q : 0)) * n;
        double out[D2_J][4];
        if constexpr (COMP) {
            // FP32 products accumulated with FMA over runs of 8 elements, each
            // run folded into a compensated (TwoSum) FP32 accumulator
            Acc2f acc[D2_J][4];
#pragma unroll
            for (int q = 0; q < D2_J; q++)
#pragma unroll
                for (int r = 0; r < 4; r++) acc[q][r].zero();
            long long e = e0 + lane;
            while (e < e1) {
                float run[D2_J][4];
#pragma unroll
                for (int q = 0; q < D2_J; q++)
#pragma unroll
                    for (int r = 0; r < 4; r++) run[q][r] = 0.f;
#pragma unroll 2
                for (int t = 0; t < 8 && e < e1; t++, e += 32) {
                    const CV uu = u[e], ww = w[e];
#pragma unroll
                    for (int q = 0; q < D2_J; q++) {
                        if (q < jn) {
                            const CV a = __ldcs(vj[q] + e);
                            run[q][0] = fmaf(a.x, uu.x, fmaf(a.y, uu.y, run[q][0]));
                            run[q][1] = fmaf(a.x, uu.y, fmaf(-a.y, uu.x, run[q][1]));
                            run[q][2] = fmaf(a.x, ww.x, fmaf(a.y, ww.y, run[q][2]));
                            run[q][3] = fmaf(a.x, ww.y, fmaf(-a.y, ww.x, run[q][3]));
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < D2_J; q++)
#pragma unroll
                    for (int r = 0; r < 4; r++) acc[q][r].add(run[q][r]);
            }
#pragma unroll
            for (int q = 0; q < D2_J; q++)
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    Acc2f t = warp_sum(acc[q][r]);
                    out[q][r] = (double)t.hi + (double)t.lo;
                }
        } else {
            typedef typename real_of<CV>::type R;
            R acc[D2_J][4];
#pragma unroll
            for (int q = 0; q < D2_J; q++)
#pragma unroll
                for (int r = 0; r < 4; r++) acc[q][r] = 0;
            long long e = e0 + lane;
            for (; e + 32 * (U - 1) < e1; e += 32 * U) {
                CV uu[U], ww[U];
#pragma unroll
                for (int t = 0; t < U; t++) {
                    uu[t] = u[e + 32 * t];
                    ww[t] = w[e + 32 * t];
                }
#pragma unroll
                for (int q = 0; q < D2_J; q++) {
                    if (q < jn) {
                        CV a[U];
#pragma unroll
                        for (int t = 0; t < U; t++) a[t] = __ldcs(vj[q] + e + 32 * t);
#pragma unroll
                        for (int t = 0; t < U; t++) {
                            acc[q][0] += a[t].x * uu[t].x + a[t].y * uu[t].y;
                            acc[q][1] += a[t].x * uu[t].y - a[t].y * uu[t].x;
                            acc[q][2] += a[t].x * ww[t].x + a[t].y * ww[t].y;
                            acc[q][3] += a[t].x * ww[t].y - a[t].y * ww[t].x;
                        }
                    }
                }
            }
            for (; e < e1; e += 32) {
                const CV u0 = u[e], w0 = w[e];
#pragma unroll
                for (int q = 0; q < D2_J; q++) {
                    if (q < jn) {
                        const CV a0 = __ldcs(vj[q] + e);
                        acc[q][0] += a0.x * u0.x + a0.y * u0.y;
                        acc[q][1] += a0.x * u0.y - a0.y * u0.x;
                        acc[q][2] += a0.x * w0.x + a0.y * w0.y;
                        acc[q][3] += a0.x * w0.y - a0.y * w0.x;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < D2_J; q++)
#pragma unroll
                for (int r = 0; r < 4; r++) out[q][r] = warp_sum((double)acc[q][r]);
        }
        if (lane == 0) {
            for (int q = 0; q < jn; q++) {
                double *p = kp.part + 4 * ((size_t)blockIdx.x * pld + (size_t)sl * nj + j0 + q);
                p[0] = out[q][0];
                p[1] = out[q][1];
                p[2] = out[q][2];
                p[3] = out[q][3];
            }
        }
    }
    if (last_block2(&st->counter[3])) {
        // warp per coefficient, lanes stride the block partials, fixed-order butterfly
        const int nparts = (int)gridDim.x * S;
        for (int j = warp; j < nj; j += D2_WARPS) {
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            for (int pi = lane; pi < nparts; pi += 32) {
                const int b = pi / S, sl = pi % S;
                const double *p = kp.part + 4 * ((size_t)b * pld + (size_t)sl * nj + j);
                s0 += __ldcg(p);
                s1 += __ldcg(p + 1);
                s2 += __ldcg(p + 2);
                s3 += __ldcg(p + 3);
            }
            s0 = warp_sum(s0);
            s1 = warp_sum(s1);
            s2 = warp_sum(s2);
            s3 = warp_sum(s3);
            if (lane == 0) {
                kp.D1[j] = make_double2(s0, s1);
                kp.D2[j] = make_double2(s2, s3);
            }
        }
    }
}

// ------------------------------------------------------------- the step
// Block sums of four values with one pair of barriers (fixed order).
static __device__ __forceinline__ void block_sum4(double &a, double &b, double &c, double &d, double (*red)[4]) {
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    d = warp_sum(d);
    if ((threadIdx.x & 31) == 0) {
        double *r = red[threadIdx.x >> 5];
        r[0] = a, r[1] = b, r[2] = c, r[3] = d;
    }
    __syncthreads();
    a = b = c = d = 0.0;
    for (int i = 0; i < STEP_THREADS / 32; i++) a += red[i][0], b += red[i][1], c += red[i][2], d += red[i][3];
}

// One block: normalisation of q_k, column k-1 of H, Givens update, residual
// estimate, stop decision and the coefficients of the axpy pass.
__global__ void __launch_bounds__(STEP_THREADS) k_dcgs2_step(KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    DevState *st = kp.st;
    if (st->stop) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red[STEP_THREADS / 32][4];
    __shared__ int flag;
    const int k = st->k;
    const double alpha = kp.D1[k].x;  // loaded ahead of the reductions
    const double2 d = kp.D2[k];
    const int ld = kp.mcap + 1;
    const int tid = threadIdx.x;
    double2 *col = reinterpret_cast<double2 *>(smraw);  // k+1 entries
    double2 *css = col + (kp.mcap + 2);                // k entries
    double *sns = reinterpret_cast<double *>(css + (kp.mcap + 1));
    double sa = 0.0, acr = 0.0, aci = 0.0, hn = 0.0;
    for (int j = tid; j < k; j += STEP_THREADS) {
        const double2 a = kp.D1[j], c = kp.D2[j];
        sa += a.x * a.x + a.y * a.y;
        acr += a.x * c.x + a.y * c.y;  // conj(a) c
        aci += a.x * c.y - a.y * c.x;
        const double2 h = cadd(kp.tv[j], a);  // column k-1 of H above the subdiagonal
        hn += h.x * h.x + h.y * h.y;
    }
    block_sum4(sa, acr, aci, hn, red);
    double nu2 = alpha - sa;
    if (tid == 0) {
        flag = (!isfinite(nu2) || !isfinite(acr) || !isfinite(aci) || !isfinite(d.x) || !isfinite(d.y) ||
                !isfinite(hn)) ? 2 : 0;
    }
    __syncthreads();
    if (flag) {
        if (tid == 0) {
            st->status = 4;
            st->stop = 1;
        }
        return;
    }
    if (!(nu2 > 0.0)) nu2 = 0.0;
    // (happy) breakdown: the new direction vanishes against the column it closes
    const bool brk = k >= 1 ? !(nu2 > 1e-28 * (hn + nu2)) : !(nu2 > 0.0);
    const double nu = sqrt(nu2);
    const double inu = nu > 0.0 ? 1.0 / nu : 0.0;
    const double2 delta = make_double2((d.x - acr) * inu, (d.y - aci) * inu);
    if (k >= 1) {
        // column k-1 of H = t + a (rows 0..k-1), nu (row k); H is stored row-major
        for (int i = tid; i < k; i += STEP_THREADS) {
            const double2 h = cadd(kp.tv[i], kp.D1[i]);
            col[i] = h;
            kp.Hm[(size_t)i * ld + (k - 1)] = h;
        }
        if (tid == 0) {
            col[k] = make_double2(nu, 0.0);
            kp.Hm[(size_t)k * ld + (k - 1)] = make_double2(nu, 0.0);
        }
        for (int j = tid; j < k - 1; j += STEP_THREADS) {
            css[j] = kp.cs[j];
            sns[j] = kp.sn[j];
        }
    }
    __syncthreads();
    // axpy coefficients P = a / nu, S = c / nu - delta a / nu^2; t_k is finished by k_axpy2
    for (int i = tid; i < k; i += STEP_THREADS) {
        const double2 a = kp.D1[i], c = kp.D2[i];
        kp.P[i] = make_double2(a.x * inu, a.y * inu);
        const double2 da = cmul(delta, a);
        kp.S[i] = make_double2((c.x - da.x * inu) * inu, (c.y - da.y * inu) * inu);
    }
    // Rotations 0..k-2 applied to col[0..k-1]: the carried entry follows the
    // affine recurrence carry_{j+1} = -s_j carry_j + c_j col[j+1], so the chain
    // is a prefix scan of affine maps.  Each thread folds a segment of the
    // rotations, the block scans the segment maps (Hillis-Steele, log2 of the
    // thread count rounds), then each thread replays its segment from its
    // incoming carry and writes the rotated entries of column k-1 into Rm.
    __shared__ double scan_a[STEP_THREADS];
    __shared__ double2 scan_b[STEP_THREADS];
    __shared__ double2 carry_last;
    const bool ref = st->rotation == 1;
    if (k >= 1) {
        const int nr = k - 1;
        const int seg = (nr + STEP_THREADS - 1) / STEP_THREADS;
        const int j0 = tid * seg < nr ? tid * seg : nr;
        const int j1 = j0 + seg < nr ? j0 + seg : nr;
        double a = 1.0;
        double2 b = make_double2(0.0, 0.0);
        for (int j = j0; j < j1; j++) {
            const double sj = sns[j];
            a = -sj * a;
            b = cadd(cscale(b, -sj), cmul(css[j], col[j + 1]));
        }
        scan_a[tid] = a;
        scan_b[tid] = b;
        __syncthreads();
        for (int off = 1; off < STEP_THREADS; off <<= 1) {
            const double a2 = scan_a[tid];
            const double2 b2 = scan_b[tid];
            const double a1 = tid >= off ? scan_a[tid - off] : 1.0;
            const double2 b1 = tid >= off ? scan_b[tid - off] : make_double2(0.0, 0.0);
            __syncthreads();
            if (tid >= off) {  // the earlier map (a1, b1), then this one (a2, b2)
                scan_a[tid] = a2 * a1;
                scan_b[tid] = cadd(cscale(b1, a2), b2);
            }
            __syncthreads();
        }
        double2 carry = col[0];
        if (tid > 0) carry = cadd(cscale(col[0], scan_a[tid - 1]), scan_b[tid - 1]);
        for (int j = j0; j < j1; j++) {
            const double2 nx = col[j + 1];
            const double2 c = css[j];
            const double sj = sns[j];
            kp.Rm[(size_t)(k - 1) * ld + j] = cadd(cmul(ref ? c : cconj(c), carry), cscale(nx, sj));
            carry = csub(cmul(c, nx), cscale(carry, sj));
        }
        if (nr == 0 ? tid == 0 : (j0 < j1 && j1 == nr)) carry_last = carry;
        __syncthreads();
    }
    if (tid == 0) {
        if (brk) st->brk = 1;
        st->cu = inu;
        st->cw = inu;
        st->du = make_double2(-delta.x * inu * inu, -delta.y * inu * inu);
        st->delta = delta;
        int stop = 0;
        if (k == 0) {
            kp.g[0] = make_double2(nu, 0.0);
        } else {
            // new rotation from (rotated col[k-1], nu)
            const double2 carry = carry_last;
            const double rho = hypot(hypot(carry.x, carry.y), nu);
            double2 c;
            double s;
            if (!(rho > 0.0) || !isfinite(rho)) {
                c = make_double2(1.0, 0.0);
                s = 0.0;
            } else {
                c = make_double2(carry.x / rho, carry.y / rho);
                s = nu / rho;
            }
            const double2 cc = ref ? c : cconj(c);
            kp.Rm[(size_t)(k - 1) * ld + (k - 1)] = cadd(cmul(cc, carry), make_double2(s * nu, 0.0));
            kp.cs[k - 1] = c;
            kp.sn[k - 1] = s;
            const double2 gk = kp.g[k - 1];
            kp.g[k] = cscale(gk, -s);
            kp.g[k - 1] = cmul(cc, gk);
            const int it = st->it + 1;
            st->it = it;
            const double gabs = hypot(gk.x, gk.y) * s;
            st->est = gabs / st->nb;
            kp.hist[it] = st->est;
            st->ncol = k;
            if (!st->fixed && (gabs <= st->tol * st->nb || gabs <= st->inner_tol * st->beta0)) stop = 1;
            if (k >= st->m) stop = 1;
            if (it >= st->maxit) stop = 1;
        }
        if (brk) stop = 1;
        st->k = k + 1;
        st->stop = stop;
    }
}

// --------------------------------------------------------------- axpy2
// q_k = cu u - sum_j P_j q_j into V[k];  u_{k+1} = cw w + du u - sum_j S_j q_j into V[k+1]
// (k = st->k - 1: the step kernel has advanced the index).
// Shared prologue of the axpy passes: P, S coefficients into shared memory
// and t_k = ([c; delta] - H(0:k, 0:k-1) a) / nu (one warp per row of H).
template <typename CV>
__device__ __forceinline__ void axpy2_prologue(const KrylovPtrs &kp, const DevState *st, int k, CV *Pc, CV *Sc) {
    typedef typename real_of<CV>::type R;
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        const double2 p = kp.P[j], q = kp.S[j];
        Pc[j] = mk<CV>((R)p.x, (R)p.y);
        Sc[j] = mk<CV>((R)q.x, (R)q.y);
    }
    const int ld = kp.mcap + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double inu = st->cu;
    for (int i = blockIdx.x * (AX2_THREADS / 32) + warp; i <= k; i += gridDim.x * (AX2_THREADS / 32)) {
        double er = 0.0, ei = 0.0;
        for (int j = (i > 0 ? i - 1 : 0) + lane; j < k; j += 32) {
            const double2 h = kp.Hm[(size_t)i * ld + j];
            const double2 a = kp.D1[j];
            er += h.x * a.x - h.y * a.y;
            ei += h.x * a.y + h.y * a.x;
        }
        er = warp_sum(er);
        ei = warp_sum(ei);
        if (lane == 0) {
            const double2 c = i < k ? kp.D2[i] : st->delta;
            kp.tv[i] = make_double2((c.x - er) * inu, (c.y - ei) * inu);
        }
    }
    __syncthreads();
}

// Tile-major axpy pass: each warp owns tiles of 32*U elements and streams the
// basis vectors over the tile with the next vector's tile in flight while
// the current one is accumulated into both outputs.
template <typename CV, int U>
__global__ void __launch_bounds__(AX2_THREADS, 2) k_axpy2t(CV *__restrict__ V, long long n, KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    V = sys_vec(V, kp);
    typedef typename real_of<CV>::type R;
    typedef typename scalar_of<CV>::type CS;
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k - 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    CS *Pc = reinterpret_cast<CS *>(smraw);
    CS *Sc = Pc + (kp.mcap + 1);
    axpy2_prologue<CS>(kp, st, k, Pc, Sc);
    const R cu = (R)st->cu, cw = (R)st->cw;
    const CS du = mk<CS>((R)st->du.x, (R)st->du.y);
    CV *u = V + (long long)k * n;
    CV *w = V + (long long)(k + 1) * n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long TILE = 32LL * U;
    const long long ntile = (n + TILE - 1) / TILE;
    const long long nw = (long long)gridDim.x * (AX2_THREADS / 32);
    for (long long tile = (long long)blockIdx.x * (AX2_THREADS / 32) + warp; tile < ntile; tile += nw) {
        const long long e0 = tile * TILE + lane;
        const bool full = tile * TILE + TILE <= n;
        CV sp[U], ss[U], a[U];
#pragma unroll
        for (int t = 0; t < U; t++) {
            sp[t] = czero<CV>();
            ss[t] = czero<CV>();
            const long long e = e0 + 32 * t;
            a[t] = (k > 0 && (full || e < n)) ? __ldcs(V + e) : czero<CV>();
        }
        for (int j = 0; j < k; j++) {
            const CS p = Pc[j], q = Sc[j];
            CV nx[U];
            const bool more = j + 1 < k;
#pragma unroll
            for (int t = 0; t < U; t++) {
                const long long e = e0 + 32 * t;
                nx[t] = (more && (full || e < n)) ? __ldcs(V + (long long)(j + 1) * n + e) : czero<CV>();
            }
#pragma unroll
            for (int t = 0; t < U; t++) {
                sp[t] = cadd(sp[t], cmul(p, a[t]));
                ss[t] = cadd(ss[t], cmul(q, a[t]));
                a[t] = nx[t];
            }
        }
#pragma unroll
        for (int t = 0; t < U; t++) {
            const long long e = e0 + 32 * t;
            if (full || e < n) {
                const CV uu = u[e], ww = w[e];
                u[e] = csub(cscale(uu, cu), sp[t]);
                w[e] = csub(cadd(cscale(ww, cw), cmul(du, uu)), ss[t]);
            }
        }
    }
}

// Split variant of the axpy pass for grids with few tiles and many basis
// vectors: a block owns a tile of 32*U elements at a time, its warps take the
// basis vectors j = w mod warps and keep partial sums of both outputs in
// registers; the partials meet in shared memory and are summed over the warps
// in a fixed order by the threads that finish the tile's elements.
// Shared memory: P, S coefficients (2 (mcap+1) elements) + 2 * warps * 32U elements.
template <typename CV, int U>
__global__ void __launch_bounds__(AX2_THREADS) k_axpy2s(CV *__restrict__ V, long long n, KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    V = sys_vec(V, kp);
    typedef typename real_of<CV>::type R;
    constexpr int W = AX2_THREADS / 32;
    constexpr int TILE = 32 * U;
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k - 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    CV *Pc = reinterpret_cast<CV *>(smraw);
    CV *Sc = Pc + (kp.mcap + 1);
    CV *red = Sc + (kp.mcap + 1);  // [W][2][TILE]
    axpy2_prologue<CV>(kp, st, k, Pc, Sc);
    const R cu = (R)st->cu, cw = (R)st->cw;
    const CV du = mk<CV>((R)st->du.x, (R)st->du.y);
    CV *u = V + (long long)k * n;
    CV *w = V + (long long)(k + 1) * n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long ntile = (n + TILE - 1) / TILE;
    for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const long long e0 = tile * TILE + lane;
        const bool full = tile * TILE + TILE <= n;
        CV sp[U], ss[U], a[U];
#pragma unroll
        for (int t = 0; t < U; t++) {
            sp[t] = czero<CV>();
            ss[t] = czero<CV>();
            const long long e = e0 + 32 * t;
            a[t] = (warp < k && (full || e < n)) ? __ldcs(V + (long long)warp * n + e) : czero<CV>();
        }
        for (int j = warp; j < k; j += W) {
            const CV p = Pc[j], q = Sc[j];
            CV nx[U];
            const bool more = j + W < k;
#pragma unroll
            for (int t = 0; t < U; t++) {
                const long long e = e0 + 32 * t;
                nx[t] = (more && (full || e < n)) ? __ldcs(V + (long long)(j + W) * n + e) : czero<CV>();
            }
#pragma unroll
            for (int t = 0; t < U; t++) {
                sp[t] = cadd(sp[t], cmul(p, a[t]));
                ss[t] = cadd(ss[t], cmul(q, a[t]));
                a[t] = nx[t];
            }
        }
#pragma unroll
        for (int t = 0; t < U; t++) {
            red[(warp * 2) * TILE + lane + 32 * t] = sp[t];
            red[(warp * 2 + 1) * TILE + lane + 32 * t] = ss[t];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < TILE; i += blockDim.x) {
            const long long e = tile * TILE + i;
            if (e < n) {
                CV s1 = czero<CV>(), s2 = czero<CV>();
#pragma unroll
                for (int wq = 0; wq < W; wq++) {
                    s1 = cadd(s1, red[(wq * 2) * TILE + i]);
                    s2 = cadd(s2, red[(wq * 2 + 1) * TILE + i]);
                }
                const CV uu = u[e], ww = w[e];
                u[e] = csub(cscale(uu, cu), s1);
                w[e] = csub(cadd(cscale(ww, cw), cmul(du, uu)), s2);
            }
        }
        __syncthreads();
    }
}

template <typename CV, int JU>
__global__ void __launch_bounds__(AX2_THREADS) k_axpy2(CV *__restrict__ V, long long n, KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    V = sys_vec(V, kp);
    typedef typename real_of<CV>::type R;
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k - 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    CV *Pc = reinterpret_cast<CV *>(smraw);
    CV *Sc = Pc + (kp.mcap + 1);
    axpy2_prologue<CV>(kp, st, k, Pc, Sc);
    const R cu = (R)st->cu, cw = (R)st->cw;
    const CV du = mk<CV>((R)st->du.x, (R)st->du.y);
    CV *u = V + (long long)k * n;
    CV *w = V + (long long)(k + 1) * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const CV uu = u[e], ww = w[e];
        CV sp = czero<CV>(), ss = czero<CV>();
        int j = 0;
        for (; j + JU <= k; j += JU) {
            CV q[JU];
#pragma unroll
            for (int t = 0; t < JU; t++) q[t] = __ldcs(V + (long long)(j + t) * n + e);
#pragma unroll
            for (int t = 0; t < JU; t++) {
                sp = cadd(sp, cmul(Pc[j + t], q[t]));
                ss = cadd(ss, cmul(Sc[j + t], q[t]));
            }
        }
        for (; j < k; j++) {
            const CV q0 = __ldcs(V + (long long)j * n + e);
            sp = cadd(sp, cmul(Pc[j], q0));
            ss = cadd(ss, cmul(Sc[j], q0));
        }
        u[e] = csub(cscale(uu, cu), sp);
        w[e] = csub(cadd(cscale(ww, cw), cmul(du, uu)), ss);
    }
}

// ------------------------------------------------------------- launchers
// Shapes of the two streaming passes.  Dot pass: 0-4 = (J, U) of the
// group-major k_dots2, 5, 6 = tile-major k_dots2t with U = 4, 8, 7, 8 = split
// k_dots2s with U = 8, 4, 9 = tile-major with U = 16 for FP32 (8 for FP64),
// 10 = tile-major with U = 14 for FP32 (7 for FP64), 11, 12 = FP32 tile-major
// on 16-byte pairs (float4 loads) with 16, 14 points per lane (even n; FP64: 6, 10).
// Axpy pass: 0-2 = j-unroll 4, 2, 8 of the element-major k_axpy2, 3, 4 =
// tile-major k_axpy2t with U = 4, 8, 5, 6 = split k_axpy2s with U = 4, 2,
// 7, 8 = tile-major with U = 16, 14 for FP32 (8, 7 for FP64), 9, 10 = FP32
// tile-major on 16-byte pairs with 8, 14 points per lane (even n; FP64: 4, 8).
// Measured on B200:
//   N = 1024, restart 100 (300 steps, k = 0..99), ms per 300 steps:
//     FP64 dots 91.6 (shape 0), 81.0 (4), 59.4 (5), 54.3 (6, 4.9 TB/s)
//     FP32 dots 97.6 (0), 78.8 (1), 50.0 (5), 38.3 (6)
//     FP64 axpy 64.4 (0), 45.7 (3), 42.0 (4, 6.5 TB/s); FP32 axpy 35.5 (2), 24.8 (4)
//   whole solves, (dots, axpy) shapes (4, 0) / (7, 5) / (split dots and axpy with U = 2):
//     256 x 256 unrestarted FP64 (1043 steps) 0.862 / 0.614 / 1.045 s
//     256 x 256 unrestarted mixed 1.754 / 0.912 / 2.120 s
//     96 x 96 GMRES(200) FP64 (180 steps) 30.6 / 18.9 / 27.9 ms
//     512 x 512 GMRES(200) FP64 (1000 steps) 0.381 / 0.254 / 0.327 s
// Defaults: tile-major on grids with tile_major(n), widths by balanced(),
// split (7, 5) below.
// CUGMRES_DOTS2_SHAPE / CUGMRES_AXPY2_SHAPE override them (diagnostics).
static int env_shape(const char *name, int nshapes) {
    const char *e = getenv(name);
    if (!e || !*e) return -1;
    const int v = atoi(e);
    return (v >= 0 && v < nshapes) ? v : -1;
}
// The tile-major passes give each warp 32 * 8 elements, so they need about as
// many tiles as the GPU holds resident warps (two 8-warp blocks per SM; from
// 3/4 of that on: n >= 454,656 on 148 SMs, N >= 675); smaller grids use the
// split passes, whose warps share the basis vectors of one tile.  Measured
// ms per step at restart 100, tile / split: 512^2 0.179 / 0.153, 768^2
// 0.303 / 0.321, 1024^2 0.442 / 0.465.
static bool tile_major(long long n, int sms) { return 4 * n >= 3LL * sms * 2 * (D2_THREADS / 32) * 32 * 8; }
// Tile width of the tile-major passes: of two instantiated widths U (points
// per lane), the one whose busiest warp streams fewer elements, i.e. the
// smaller ceil(tiles / resident warps) * U, ties to the first.  The resident
// warps are two 8-warp blocks per SM.  At n = 2^20 on 148 SMs, U = 8 gives
// 4096 tiles over 2368 warps (the second wave 73 % full) and U = 7 gives
// 4682 (99 %); measured at 1024^2, ms per 1000 steps: FP64 dots 150.7 (U = 8)
// -> 142.2 (U = 7), FP64 axpy 140.1 -> 138.0, FP32 dots 97.8 (U = 8) -> 86.8
// (U = 16) -> 83.5 (U = 14), FP32 axpy 82.2 (U = 8) -> 78.4 (U = 14); at
// 2048^2 FP32 dots 34.3 (U = 16) -> 32.3 (U = 14), FP32 axpy 32.0 (U = 8)
// against 32.7 (U = 14, a tie by the rule).
static int balanced(long long n, int sms, int va, int Ua, int vb, int Ub) {
    const long long nw = 2LL * sms * (D2_THREADS / 32);
    auto cost = [&](int U) {
        const long long tiles = (n + 32LL * U - 1) / (32LL * U);
        return (tiles + nw - 1) / nw * U;
    };
    return cost(Ub) < cost(Ua) ? vb : va;
}
static int dots2_shape(int prec_v, long long n, int sms) {
    static const int v = env_shape("CUGMRES_DOTS2_SHAPE", 13);
    if (v >= 0) return v;
    if (!tile_major(n, sms)) return 7;
    if (prec_v == 0) return balanced(n, sms, 6, 8, 10, 7);
    return n % 2 == 0 ? balanced(n, sms, 11, 16, 12, 14) : balanced(n, sms, 9, 16, 10, 14);
}
static int axpy2_shape(int prec_v, long long n, int sms) {
    static const int v = env_shape("CUGMRES_AXPY2_SHAPE", 11);
    if (v >= 0) return v;
    if (!tile_major(n, sms)) return 5;
    if (prec_v == 0) return balanced(n, sms, 4, 8, 8, 7);
    return n % 2 == 0 ? balanced(n, sms, 9, 8, 10, 14) : balanced(n, sms, 4, 8, 8, 14);
}

template <typename CV, bool COMP> struct Dots2Table {
    typedef void (*K)(const CV *, long long, KrylovPtrs);
    static K get(int v) {
        switch (v) {
            case 1: return k_dots2<CV, COMP, 2, 2>;
            case 2: return k_dots2<CV, COMP, 4, 1>;
            case 3: return k_dots2<CV, COMP, 8, 1>;
            case 4: return k_dots2<CV, COMP, 2, 4>;
            case 5: return k_dots2t<CV, 4>;
            case 6: return k_dots2t<CV, 8>;
            case 7: return k_dots2s<CV, 8>;
            case 8: return k_dots2s<CV, 4>;
            case 9:  // 16 points per lane: the FP64 tile's bytes for FP32 vectors
                if constexpr (sizeof(CV) == 8) return k_dots2t<CV, 16>;
                else return k_dots2t<CV, 8>;
            case 10:  // 7 (FP64) / 14 (FP32) points per lane
                if constexpr (sizeof(CV) == 8) return k_dots2t<CV, 14>;
                else return k_dots2t<CV, 7>;
            // 11, 12: FP32 on even lengths runs k_dots2t<float4, 8 / 7> (dots2_vec_kernel);
            // the same widths in complex values otherwise
            case 11:
                if constexpr (sizeof(CV) == 8) return k_dots2t<CV, 16>;
                else return k_dots2t<CV, 8>;
            case 12:
                if constexpr (sizeof(CV) == 8) return k_dots2t<CV, 14>;
                else return k_dots2t<CV, 7>;
            default: return k_dots2<CV, COMP, 4, 2>;
        }
    }
};
template <typename CV> struct Axpy2Table {
    typedef void (*K)(CV *, long long, KrylovPtrs);
    static K get(int v) {
        switch (v) {
            case 1: return k_axpy2<CV, 2>;
            case 2: return k_axpy2<CV, 8>;
            case 3: return k_axpy2t<CV, 4>;
            case 4: return k_axpy2t<CV, 8>;
            case 5: return k_axpy2s<CV, 4>;
            case 6: return k_axpy2s<CV, 2>;
            case 7:  // 16 points per lane for FP32 vectors
                if constexpr (sizeof(CV) == 8) return k_axpy2t<CV, 16>;
                else return k_axpy2t<CV, 8>;
            case 8:  // 7 (FP64) / 14 (FP32) points per lane
                if constexpr (sizeof(CV) == 8) return k_axpy2t<CV, 14>;
                else return k_axpy2t<CV, 7>;
            // 9, 10: FP32 on even lengths runs k_axpy2t<float4, 4 / 7> (axpy2_vec_kernel);
            // the same widths in complex values otherwise
            case 9: return k_axpy2t<CV, 8>;
            case 10:
                if constexpr (sizeof(CV) == 8) return k_axpy2t<CV, 14>;
                else return k_axpy2t<CV, 7>;
            default: return k_axpy2<CV, 4>;
        }
    }
};

// Dynamic shared memory of the dot-pass shapes: per-warp coefficient slots
// (tile-major) or one slot per coefficient (split), for chunks of cs vectors.
static size_t dots2_smem(int v, int mcap) {
    const int jc = mcap + 1 < D2T_CHUNK ? mcap + 1 : D2T_CHUNK;
    if (v == 5 || v == 6 || (v >= 9 && v <= 12)) return (size_t)D2_WARPS * (size_t)jc * 4 * sizeof(double);
    if (v == 7 || v == 8) return (size_t)jc * 4 * sizeof(double);
    return 0;
}

// FP32 tile-major shapes on 16-byte pairs of complex values (even n only)
static bool dots2_vec(int prec_v, long long n, int v) { return prec_v != 0 && n % 2 == 0 && (v == 11 || v == 12); }
static bool axpy2_vec(int prec_v, long long n, int v) { return prec_v != 0 && n % 2 == 0 && (v == 9 || v == 10); }
typedef void (*DotsVecK)(const float4 *, long long, KrylovPtrs);
typedef void (*AxpyVecK)(float4 *, long long, KrylovPtrs);
static DotsVecK dots2_vec_kernel(int v, size_t smem) {
    DotsVecK kern = v == 11 ? k_dots2t<float4, 8> : k_dots2t<float4, 7>;
    smem_optin(kern, smem);
    return kern;
}
static AxpyVecK axpy2_vec_kernel(int v, size_t smem) {
    AxpyVecK kern = v == 9 ? k_axpy2t<float4, 4> : k_axpy2t<float4, 7>;
    smem_optin(kern, smem);
    return kern;
}

template <typename CV, bool COMP> static typename Dots2Table<CV, COMP>::K dots2_kernel(int v, size_t smem) {
    typename Dots2Table<CV, COMP>::K kern = Dots2Table<CV, COMP>::get(v);
    smem_optin(kern, smem);
    return kern;
}

// Blocks with any work: a tile of 32*U elements per warp (tile-major) or per
// block (split); more blocks would only add partial sums to reduce.
static long long work_blocks(bool split, int U, long long n) {
    const long long tiles = (n + 32LL * U - 1) / (32LL * U);
    const long long b = split ? tiles : (tiles + D2_WARPS - 1) / D2_WARPS;
    return b < 1 ? 1 : b;
}

int dots2_blocks(int prec_v, int sms, int mcap, long long n) {
    const int v = dots2_shape(prec_v, n, sms);
    const size_t smem = dots2_smem(v, mcap);
    int g = dots2_vec(prec_v, n, v) ? waves_grid(dots2_vec_kernel(v, smem), D2_THREADS, smem, sms)
            : prec_v == 0           ? waves_grid(dots2_kernel<double2, false>(v, smem), D2_THREADS, smem, sms)
                                    : waves_grid(dots2_kernel<float2, true>(v, smem), D2_THREADS, smem, sms);
    if (v >= 5 && v <= 12) {
        // points per lane, in complex values
        const int U = (v == 5 || v == 8) ? 4
                      : (v == 10 || v == 12) ? (prec_v != 0 ? 14 : 7)
                      : ((v == 9 || v == 11) && prec_v != 0) ? 16 : 8;
        const long long cap = work_blocks(v == 7 || v == 8, U, n);
        if (cap < g) g = (int)cap;
    }
    return g;
}

int launch_dots2(int prec_v, const void *V, long long n, const KrylovPtrs &kp, int nblk, int sms, cudaStream_t s) {
    const int v = dots2_shape(prec_v, n, sms);
    const size_t smem = dots2_smem(v, kp.mcap);
    const dim3 grid(nblk, kp.nsys);
    if (dots2_vec(prec_v, n, v)) {
        KrylovPtrs kq = kp;
        kq.sys_v = kp.sys_v / 2;  // the basis in pairs of complex values
        dots2_vec_kernel(v, smem)<<<grid, D2_THREADS, smem, s>>>((const float4 *)V, n / 2, kq);
    } else if (prec_v == 0) {
        dots2_kernel<double2, false>(v, smem)<<<grid, D2_THREADS, smem, s>>>((const double2 *)V, n, kp);
    } else {
        dots2_kernel<float2, true>(v, smem)<<<grid, D2_THREADS, smem, s>>>((const float2 *)V, n, kp);
    }
    return (int)cudaGetLastError();
}

int launch_dcgs2_step(const KrylovPtrs &kp, cudaStream_t s) {
    const size_t smem = (size_t)(kp.mcap + 2) * sizeof(double2) + (size_t)(kp.mcap + 1) * sizeof(double2) +
                        (size_t)(kp.mcap + 1) * sizeof(double);
    if (int e = smem_optin(k_dcgs2_step, smem)) return e;
    k_dcgs2_step<<<dim3(1, kp.nsys), STEP_THREADS, smem, s>>>(kp);
    return (int)cudaGetLastError();
}

template <typename CV> static int axpy2_prepare(int v, size_t smem) {
    return smem_optin(Axpy2Table<CV>::get(v), smem);
}

// Dynamic shared memory of the axpy-pass shapes: P, S coefficients, plus the
// per-warp partial sums of the split shapes.
static size_t axpy2_smem(int v, int prec_v, int mcap) {
    const size_t e = prec_v == 0 ? sizeof(double2) : sizeof(float2);
    size_t b = 2 * (size_t)(mcap + 1) * e;
    if (v == 5 || v == 6) b += 2 * (size_t)(AX2_THREADS / 32) * 32 * (v == 5 ? 4 : 2) * e;
    return b;
}

int axpy2_blocks(int prec_v, int sms, int mcap, long long n) {
    const int v = axpy2_shape(prec_v, n, sms);
    const size_t smem = axpy2_smem(v, prec_v, mcap);
    int g;
    if (axpy2_vec(prec_v, n, v)) {
        g = waves_grid(axpy2_vec_kernel(v, smem), AX2_THREADS, smem, sms);
    } else if (prec_v == 0) {
        axpy2_prepare<double2>(v, smem);
        g = waves_grid(Axpy2Table<double2>::get(v), AX2_THREADS, smem, sms);
    } else {
        axpy2_prepare<float2>(v, smem);
        g = waves_grid(Axpy2Table<float2>::get(v), AX2_THREADS, smem, sms);
    }
    if (v >= 3 && v <= 10) {
        // points per lane, in complex values
        const int U = (v == 3 || v == 5) ? 4
                      : (v == 4 || v == 9) ? 8
                      : v == 6 ? 2
                      : (v == 8 || v == 10) ? (prec_v != 0 ? 14 : 7)
                                            : (prec_v != 0 ? 16 : 8);
        const long long cap = work_blocks(v == 5 || v == 6, U, n);
        if (cap < g) g = (int)cap;
    }
    return g;
}

int launch_axpy2(int prec_v, const void *V, long long n, const KrylovPtrs &kp, int nblk, int sms, cudaStream_t s) {
    const int v = axpy2_shape(prec_v, n, sms);
    const size_t smem = axpy2_smem(v, prec_v, kp.mcap);
    const dim3 grid(nblk, kp.nsys);
    if (axpy2_vec(prec_v, n, v)) {
        KrylovPtrs kq = kp;
        kq.sys_v = kp.sys_v / 2;  // the basis in pairs of complex values
        axpy2_vec_kernel(v, smem)<<<grid, AX2_THREADS, smem, s>>>((float4 *)V, n / 2, kq);
        return (int)cudaGetLastError();
    }
    int e = prec_v == 0 ? axpy2_prepare<double2>(v, smem) : axpy2_prepare<float2>(v, smem);
    if (e) return e;
    if (prec_v == 0) Axpy2Table<double2>::get(v)<<<grid, AX2_THREADS, smem, s>>>((double2 *)V, n, kp);
    else Axpy2Table<float2>::get(v)<<<grid, AX2_THREADS, smem, s>>>((float2 *)V, n, kp);
    return (int)cudaGetLastError();
}

}  // namespace cg
