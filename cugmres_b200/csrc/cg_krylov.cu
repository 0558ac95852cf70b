// Arnoldi (CGS2) and least-squares kernels of the GMRES cycle.
//
// Reference behaviour (CUDA_GMRES/GMRES.cuh:289-371): modified Gram-Schmidt
// with one cublasCdotc and one weight_subtract_kernel launch per basis vector,
// cublasScnrm2 + Csscal for the new vector, two cublasCgemm3m on explicit
// (m+1)^2 Givens matrices per iteration and a host round trip for the residual.
//
// Here one Arnoldi step is classical Gram-Schmidt with one
// reorthogonalisation (CGS2) in four bandwidth-bound passes over the basis:
//   k_dots   h1 = V^H w          (all basis vectors in one launch)
//   k_axpy   w -= V h1
//   k_dots   h2 = V^H w
//   k_axpy   w -= V h2, ||w||^2 fused
// followed by k_givens, one warp that applies the stored rotations to the new
// Hessenberg column, makes the next rotation, updates the residual estimate and
// decides on device whether the cycle continues.  Basis vectors are stored
// unnormalised with a per-vector scale (scale[j] = 1/||w_j||), which every
// reader applies, so normalisation costs no extra pass.  Reductions are
// deterministic: fixed per-block partitions, fixed-order warp butterflies and a
// last-block fixed-order sum over block partials.
#include "cg_common.cuh"
#include "cg_internal.h"

namespace cg {

static constexpr int DOT_THREADS = 256;
static constexpr int AXPY_THREADS = 256;

static __device__ __forceinline__ void block_range(long long n, int nblk, int blk, long long &e0, long long &e1) {
    long long chunk = (n + nblk - 1) / nblk;
    chunk = (chunk + 127) & ~127LL;
    e0 = (long long)blk * chunk;
    if (e0 > n) e0 = n;
    e1 = e0 + chunk;
    if (e1 > n) e1 = n;
}

// Returns true in exactly one block: the last one to finish (after all others
// made their partials visible).  Resets the ticket for the next launch.
static __device__ __forceinline__ bool last_block(unsigned int *ticket) {
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

// ------------------------------------------------------------------ dots
// out[j] = scale[j] * sum_e conj(V_j[e]) w[e], j = 0..k (k = st->k).
// Each warp owns basis vectors j = warp, warp+8, ...; lanes stride the block's
// element range; w is re-read from L1 for every vector.
template <typename CV, typename CW, bool COMP>
__global__ void __launch_bounds__(DOT_THREADS)
k_dots(const CV *__restrict__ V, long long n, KrylovPtrs kp, VecSel w, double2 *__restrict__ out, int ctr, int gate) {
    kp = kp_sys(kp);  // this block's system of a bucket
    V = sys_vec(V, kp);
    DevState *st = kp.st;
    if (gate == GATE_STOP && st->stop) return;
    const int nj = st->k + 1;
    const CW *wv = reinterpret_cast<const CW *>(w.base) + (long long)(st->k + w.koff) * w.stride +
                   (long long)blockIdx.y * w.sys;
    out = sys_move_bytes(out, kp.sys_ws);
    long long e0, e1;
    block_range(n, gridDim.x, blockIdx.x, e0, e1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ld = kp.mcap + 1;
    for (int j = warp; j < nj; j += DOT_THREADS / 32) {
        const CV *vj = V + (long long)j * n;
        double re, im;
        if constexpr (COMP) {
            Acc2f ar[2], ai[2];
            ar[0].zero(); ar[1].zero(); ai[0].zero(); ai[1].zero();
            long long e = e0 + lane;
            for (; e + 32 < e1; e += 64) {
                const CV a0 = vj[e], a1 = vj[e + 32];
                const CW b0 = wv[e], b1 = wv[e + 32];
                ar[0].add_prod(a0.x, b0.x); ar[0].add_prod(a0.y, b0.y);
                ai[0].add_prod(a0.x, b0.y); ai[0].add_prod(-a0.y, b0.x);
                ar[1].add_prod(a1.x, b1.x); ar[1].add_prod(a1.y, b1.y);
                ai[1].add_prod(a1.x, b1.y); ai[1].add_prod(-a1.y, b1.x);
            }
            if (e < e1) {
                const CV a0 = vj[e];
                const CW b0 = wv[e];
                ar[0].add_prod(a0.x, b0.x); ar[0].add_prod(a0.y, b0.y);
                ai[0].add_prod(a0.x, b0.y); ai[0].add_prod(-a0.y, b0.x);
            }
            ar[0].add_acc(ar[1]);
            ai[0].add_acc(ai[1]);
            Acc2f sr = warp_sum(ar[0]), si = warp_sum(ai[0]);
            re = (double)sr.hi + (double)sr.lo;
            im = (double)si.hi + (double)si.lo;
        } else {
            typedef typename real_of<CW>::type R;
            R r0 = 0, r1 = 0, r2 = 0, r3 = 0, i0 = 0, i1 = 0, i2 = 0, i3 = 0;
            long long e = e0 + lane;
            for (; e + 96 < e1; e += 128) {
                const CV a0 = vj[e], a1 = vj[e + 32], a2 = vj[e + 64], a3 = vj[e + 96];
                const CW b0 = wv[e], b1 = wv[e + 32], b2 = wv[e + 64], b3 = wv[e + 96];
                r0 += a0.x * b0.x + a0.y * b0.y; i0 += a0.x * b0.y - a0.y * b0.x;
                r1 += a1.x * b1.x + a1.y * b1.y; i1 += a1.x * b1.y - a1.y * b1.x;
                r2 += a2.x * b2.x + a2.y * b2.y; i2 += a2.x * b2.y - a2.y * b2.x;
                r3 += a3.x * b3.x + a3.y * b3.y; i3 += a3.x * b3.y - a3.y * b3.x;
            }
            for (; e < e1; e += 32) {
                const CV a0 = vj[e];
                const CW b0 = wv[e];
                r0 += a0.x * b0.x + a0.y * b0.y; i0 += a0.x * b0.y - a0.y * b0.x;
            }
            re = warp_sum((double)((r0 + r1) + (r2 + r3)));
            im = warp_sum((double)((i0 + i1) + (i2 + i3)));
        }
        if (lane == 0) {
            double *p = kp.part + 2 * ((size_t)blockIdx.x * ld + j);
            p[0] = re;
            p[1] = im;
        }
    }
    if (last_block(&st->counter[ctr])) {
        // warp per coefficient, lanes stride the block partials, fixed-order butterfly
        for (int j = warp; j < nj; j += DOT_THREADS / 32) {
            double re = 0.0, im = 0.0;
            for (int b = lane; b < (int)gridDim.x; b += 32) {
                const double *p = kp.part + 2 * ((size_t)b * ld + j);
                re += __ldcg(p);
                im += __ldcg(p + 1);
            }
            re = warp_sum(re);
            im = warp_sum(im);
            if (lane == 0) {
                const double s = kp.scale[j];
                out[j] = make_double2(re * s, im * s);
            }
        }
    }
}

// ------------------------------------------------------------------ axpy
// w[e] += sum_j coef_j V_j[e], coef_j = sign * scale[j] * src[j], for
// j < nj (nj = k+1 or k).  Optionally accumulates ||w||^2 into st->wnorm2.
template <typename CV, typename CW>
__global__ void __launch_bounds__(AXPY_THREADS)
k_axpy(const CV *__restrict__ V, long long n, KrylovPtrs kp, const double2 *__restrict__ src, double sign, int nj_mode,
       VecSel w, int want_norm, int ctr, int gate) {
    kp = kp_sys(kp);  // this block's system of a bucket
    V = sys_vec(V, kp);
    typedef typename real_of<CW>::type R;
    DevState *st = kp.st;
    if (gate == GATE_STOP && st->stop) return;
    const int nj = (nj_mode == NJ_K_PLUS_1) ? st->k + 1 : (nj_mode == NJ_K ? st->k : st->ncol);
    src = sys_move_bytes(src, kp.sys_ws);
    extern __shared__ __align__(16) unsigned char smraw[];
    CW *coef = reinterpret_cast<CW *>(smraw);
    __shared__ double wsum[AXPY_THREADS / 32];
    for (int j = threadIdx.x; j < nj; j += blockDim.x) {
        const double2 v = src[j];
        const double s = sign * kp.scale[j];
        coef[j] = mk<CW>((R)(v.x * s), (R)(v.y * s));
    }
    __syncthreads();
    CW *wv = reinterpret_cast<CW *>(w.base) + (long long)(st->k + w.koff) * w.stride + (long long)blockIdx.y * w.sys;
    double nrm = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        CW acc = wv[e];
        int j = 0;
        for (; j + 4 <= nj; j += 4) {
            const CV a0 = V[(long long)j * n + e];
            const CV a1 = V[(long long)(j + 1) * n + e];
            const CV a2 = V[(long long)(j + 2) * n + e];
            const CV a3 = V[(long long)(j + 3) * n + e];
            const CW c0 = coef[j], c1 = coef[j + 1], c2 = coef[j + 2], c3 = coef[j + 3];
            acc.x += c0.x * a0.x - c0.y * a0.y; acc.y += c0.x * a0.y + c0.y * a0.x;
            acc.x += c1.x * a1.x - c1.y * a1.y; acc.y += c1.x * a1.y + c1.y * a1.x;
            acc.x += c2.x * a2.x - c2.y * a2.y; acc.y += c2.x * a2.y + c2.y * a2.x;
            acc.x += c3.x * a3.x - c3.y * a3.y; acc.y += c3.x * a3.y + c3.y * a3.x;
        }
        for (; j < nj; j++) {
            const CV a0 = V[(long long)j * n + e];
            const CW c0 = coef[j];
            acc.x += c0.x * a0.x - c0.y * a0.y; acc.y += c0.x * a0.y + c0.y * a0.x;
        }
        wv[e] = acc;
        nrm += (double)acc.x * (double)acc.x + (double)acc.y * (double)acc.y;
    }
    if (want_norm) {
        nrm = warp_sum(nrm);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = nrm;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int i = 0; i < AXPY_THREADS / 32; i++) t += wsum[i];
            kp.npart[blockIdx.x] = t;
        }
        if (last_block(&st->counter[ctr])) {
            if (threadIdx.x < 32) {
                double t = 0.0;
                for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) t += __ldcg(kp.npart + b);
                t = warp_sum(t);
                if (threadIdx.x == 0) st->wnorm2 = t;
            }
        }
    }
}

// ---------------------------------------------------------------- givens
// One warp.  New Hessenberg column h = h1 + h2 (and ||w|| below it): apply
// the stored rotations j < k, make rotation k, rotate g, record the estimate
// and decide whether the cycle stops.  Rotation formulas:
//   unitary   [[conj(c), s], [-s, c]],  c = a/rho, s = |w|/rho
//   reference [[c, s], [-s, c]]  (MKL_GMRES_test_09122019/source/loop_functions.h:630-689,
//             J(i,i) = J(i+1,i+1) = Htemp(i,i)/rho, J(i,i+1) = Htemp(i+1,i)/rho,
//             J(i+1,i) = -conj(Htemp(i+1,i))/rho).
__global__ void k_givens(KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k;
    const int ld = kp.mcap + 1;
    const int lane = threadIdx.x;
    double2 *Rk = kp.Rm + (size_t)k * ld;
    for (int j = lane; j <= k; j += 32) Rk[j] = cadd(kp.h1[j], kp.h2[j]);
    __syncwarp();
    if (lane != 0) return;
    const bool ref = st->rotation == 1;
    const double hk1 = sqrt(st->wnorm2);
    bool finite = isfinite(hk1);
    for (int j = 0; j < k; j++) {
        const double2 a = Rk[j], b = Rk[j + 1];
        const double2 c = kp.cs[j];
        const double s = kp.sn[j];
        const double2 cc = ref ? c : cconj(c);
        Rk[j] = cadd(cmul(cc, a), cscale(b, s));
        Rk[j + 1] = csub(cmul(c, b), cscale(a, s));
    }
    const double2 a = Rk[k];
    finite = finite && isfinite(a.x) && isfinite(a.y);
    const double rho = hypot(hypot(a.x, a.y), hk1);
    double2 c;
    double s;
    if (!(rho > 0.0) || !isfinite(rho)) {
        c = make_double2(1.0, 0.0);
        s = 0.0;
    } else {
        c = make_double2(a.x / rho, a.y / rho);
        s = hk1 / rho;
    }
    kp.cs[k] = c;
    kp.sn[k] = s;
    const double2 cc = ref ? c : cconj(c);
    Rk[k] = cadd(cmul(cc, a), make_double2(s * hk1, 0.0));
    const double2 gk = kp.g[k];
    kp.g[k + 1] = cscale(gk, -s);
    kp.g[k] = cmul(cc, gk);
    const int it = st->it + 1;
    st->it = it;
    const double gabs = hypot(gk.x, gk.y) * s;
    const double est = gabs / st->nb;
    st->est = est;
    kp.hist[it] = est;
    kp.scale[k + 1] = hk1 > 0.0 ? 1.0 / hk1 : 0.0;
    st->k = k + 1;
    st->ncol = k + 1;
    int stop = 0;
    if (!finite) {
        st->status = 4;
        stop = 1;
    }
    if (!(hk1 > 0.0)) {
        st->brk = 1;
        stop = 1;
    }
    if (!st->fixed && (gabs <= st->tol * st->nb || gabs <= st->inner_tol * st->beta0)) stop = 1;
    if (k + 1 >= st->m) stop = 1;
    if (it >= st->maxit) stop = 1;
    st->stop = stop;
}

// ------------------------------------------------------------ back-solve
// One warp: y = R^{-1} g for the kk = st->k columns of this cycle, column-
// oriented so the lanes update the remaining right-hand side in parallel.
__global__ void k_backsolve(KrylovPtrs kp) {
    kp = kp_sys(kp);  // this block's system of a bucket
    DevState *st = kp.st;
    const int kk = st->ncol;
    const int ld = kp.mcap + 1;
    const int lane = threadIdx.x;
    extern __shared__ __align__(16) unsigned char smraw[];
    double2 *gs = reinterpret_cast<double2 *>(smraw);
    for (int j = lane; j < kk; j += 32) gs[j] = kp.g[j];
    __syncwarp();
    for (int i = kk - 1; i >= 0; i--) {
        const double2 *Ri = kp.Rm + (size_t)i * ld;
        if (lane == 0) {
            const double2 d = Ri[i];
            const double dd = d.x * d.x + d.y * d.y;
            double2 yi = dd > 0.0 ? cscale(cmulc(d, gs[i]), 1.0 / dd) : make_double2(0.0, 0.0);
            gs[i] = yi;
            kp.y[i] = yi;
        }
        __syncwarp();
        const double2 yi = gs[i];
        for (int l = lane; l < i; l += 32) gs[l] = csub(gs[l], cmul(Ri[l], yi));
        __syncwarp();
    }
}

// ---------------------------------------------------------- cycle begin
// One warp: ||r||^2 partials of the residual pass -> beta, true residual,
// convergence / budget / breakdown decisions, reset of the cycle state.
__global__ void k_cycle_begin(KrylovPtrs kp, int nparts) {
    kp = kp_sys(kp);  // this block's system of a bucket
    DevState *st = kp.st;
    const int lane = threadIdx.x;
    double acc = 0.0;
    for (int i = lane; i < nparts; i += 32) acc += kp.npart[i];
    acc = warp_sum(acc);
    const int m = st->m;
    for (int j = lane; j <= m; j += 32) kp.g[j] = make_double2(0.0, 0.0);
    for (int j = lane; j <= m + 1; j += 32) kp.scale[j] = 1.0;
    __syncwarp();
    if (lane != 0) return;
    const double beta = sqrt(acc);
    const double rel = beta / st->nb;
    st->true_res = rel;
    st->beta0 = beta;
    if (st->cycles == 0) kp.hist[0] = rel;
    st->k = 0;
    st->ncol = 0;
    if (st->status != 0) {  // a system of a bucket that has finished stays finished
        st->stop = 1;
        return;
    }
    int stop = 0;
    if (!isfinite(beta)) {
        st->status = 4;
        stop = 1;
    } else if (st->fixed ? (beta <= st->tol) : (rel <= st->tol)) {
        st->status = 1;
        stop = 1;
    } else if (st->fixed && st->cycles > 0) {
        st->status = 2;  // reference semantics: exactly one cycle
        stop = 1;
    } else if (st->it >= st->maxit) {
        st->status = 2;
        stop = 1;
    } else if (st->brk) {
        st->status = 3;
        stop = 1;
    }
    st->brk = 0;
    if (!stop) {
        st->cycles += 1;  // cycles that run Arnoldi steps (the final check is not one)
        // CGS2 normalises V_0 lazily; the delayed scheme normalises it in its first step
        if (st->ortho == 1) kp.scale[0] = 1.0 / beta;
        kp.g[0] = make_double2(beta, 0.0);
    }
    st->stop = stop;
}

// ------------------------------------------------------------------ norm
template <typename C>
__global__ void __launch_bounds__(256) k_norm2(const C *__restrict__ v, long long n, double *npart, unsigned int *ticket,
                                               double *out) {
    __shared__ double wsum[8];
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const C a = v[e];
        acc += (double)a.x * (double)a.x + (double)a.y * (double)a.y;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < 8; i++) t += wsum[i];
        npart[blockIdx.x] = t;
    }
    if (last_block(ticket)) {
        if (threadIdx.x < 32) {
            double t = 0.0;
            for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) t += __ldcg(npart + b);
            t = warp_sum(t);
            if (threadIdx.x == 0) *out = sqrt(t);
        }
    }
}

template <typename CI, typename CO>
__global__ void k_convert(const CI *__restrict__ a, CO *__restrict__ b, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) b[e] = to_c(a[e], CO());
}

// ------------------------------------------------------------- launchers
int launch_dots(int prec_v, const void *V, long long n, const KrylovPtrs &kp, VecSel w, double2 *out, int ctr,
                int nblk, int gate, cudaStream_t s) {
    if (prec_v == 0)
        k_dots<double2, double2, false><<<dim3(nblk, kp.nsys), DOT_THREADS, 0, s>>>((const double2 *)V, n, kp, w, out, ctr, gate);
    else
        k_dots<float2, float2, true><<<dim3(nblk, kp.nsys), DOT_THREADS, 0, s>>>((const float2 *)V, n, kp, w, out, ctr, gate);
    return (int)cudaGetLastError();
}

template <typename K> static int smem_attr(K kern, size_t smem) { return smem_optin(kern, smem); }

int launch_axpy(int prec_v, int prec_w, const void *V, long long n, const KrylovPtrs &kp, const double2 *src,
                double sign, int nj_mode, VecSel w, int want_norm, int ctr, int nblk, int gate, cudaStream_t s) {
    const size_t smem = (size_t)(kp.mcap + 1) * (prec_w == 0 ? sizeof(double2) : sizeof(float2));
    int e = 0;
    if (prec_v == 0 && prec_w == 0) e = smem_attr(k_axpy<double2, double2>, smem);
    else if (prec_v == 1 && prec_w == 1) e = smem_attr(k_axpy<float2, float2>, smem);
    else if (prec_v == 1 && prec_w == 0) e = smem_attr(k_axpy<float2, double2>, smem);
    if (e) return e;
    if (prec_v == 0 && prec_w == 0)
        k_axpy<double2, double2><<<dim3(nblk, kp.nsys), AXPY_THREADS, smem, s>>>((const double2 *)V, n, kp, src, sign, nj_mode, w,
                                                                    want_norm, ctr, gate);
    else if (prec_v == 1 && prec_w == 1)
        k_axpy<float2, float2><<<dim3(nblk, kp.nsys), AXPY_THREADS, smem, s>>>((const float2 *)V, n, kp, src, sign, nj_mode, w,
                                                                  want_norm, ctr, gate);
    else if (prec_v == 1 && prec_w == 0)
        k_axpy<float2, double2><<<dim3(nblk, kp.nsys), AXPY_THREADS, smem, s>>>((const float2 *)V, n, kp, src, sign, nj_mode, w,
                                                                   want_norm, ctr, gate);
    else
        return -1;
    return (int)cudaGetLastError();
}

int launch_givens(const KrylovPtrs &kp, cudaStream_t s) {
    k_givens<<<dim3(1, kp.nsys), 32, 0, s>>>(kp);
    return (int)cudaGetLastError();
}

int launch_backsolve(const KrylovPtrs &kp, cudaStream_t s) {
    const size_t smem = (size_t)(kp.mcap + 1) * sizeof(double2);
    int e = smem_attr(k_backsolve, smem);
    if (e) return e;
    k_backsolve<<<dim3(1, kp.nsys), 32, smem, s>>>(kp);
    return (int)cudaGetLastError();
}

// Switches the orthogonalisation mode of the cycle that k_cycle_begin has just
// set up (flexible GMRES alternates preconditioned CGS2 cycles with plain
// delayed-CGS2 cycles): the only mode-specific part of a cycle's start is the
// lazy normalisation of V_0 that CGS2 keeps in scale[0].
__global__ void k_set_ortho(KrylovPtrs kp, int ortho) {
    kp = kp_sys(kp);  // this block's system of a bucket
    DevState *st = kp.st;
    st->ortho = ortho;
    if (!st->stop) kp.scale[0] = ortho == 1 ? 1.0 / st->beta0 : 1.0;
}

int launch_set_ortho(const KrylovPtrs &kp, int ortho, cudaStream_t s) {
    k_set_ortho<<<dim3(1, kp.nsys), 1, 0, s>>>(kp, ortho);
    return (int)cudaGetLastError();
}

int launch_cycle_begin(const KrylovPtrs &kp, int nparts, cudaStream_t s) {
    k_cycle_begin<<<dim3(1, kp.nsys), 32, 0, s>>>(kp, nparts);
    return (int)cudaGetLastError();
}

int launch_norm2(int prec, const void *v, long long n, double *npart, unsigned int *counter, double *out, int nblk,
                 cudaStream_t s) {
    if (prec == 0) k_norm2<double2><<<nblk, 256, 0, s>>>((const double2 *)v, n, npart, counter, out);
    else k_norm2<float2><<<nblk, 256, 0, s>>>((const float2 *)v, n, npart, counter, out);
    return (int)cudaGetLastError();
}

int launch_convert(int from_prec, int to_prec, const void *src, void *dst, long long n, cudaStream_t s) {
    const int nb = (int)((n + 255) / 256 > 4096 ? 4096 : (n + 255) / 256);
    if (from_prec == 0 && to_prec == 1) k_convert<double2, float2><<<nb, 256, 0, s>>>((const double2 *)src, (float2 *)dst, n);
    else if (from_prec == 1 && to_prec == 0) k_convert<float2, double2><<<nb, 256, 0, s>>>((const float2 *)src, (double2 *)dst, n);
    else return -1;
    return (int)cudaGetLastError();
}

}  // namespace cg
