// s-step (communication-avoiding) Arnoldi for GMRES.
//
// The delayed CGS2 step (cg_dcgs2.cu) reads the basis twice per Arnoldi step,
// which is most of a step's bytes at restart 100 (the dot and axpy passes run
// at the HBM roofline).  Here S steps are taken at once (Hoemmen, "Communication-
// avoiding Krylov subspace methods", PhD thesis, UC Berkeley 2010, ch. 3):
//
//   1. matrix powers: S matvecs build a Newton basis from the last orthonormal
//      vector q_k,  w_1 = (A - th_0) q_k,  w_{i+1} = (A - th_i) w_i,  into V[k+1..k+S]
//      (the shift is fused into the inverse row pass of each matvec);
//   2. block Gram-Schmidt with the Pythagorean Cholesky (BCGS-PIP, Barlow,
//      SIAM J. Matrix Anal. Appl. 40 (2019); Carson, Lund, Rozloznik, SIAM J.
//      Matrix Anal. Appl. 42 (2021)), twice: one pass computes C = Q^H W and the
//      Gram matrix G = W^H W together, a one-block kernel factors
//      G - C^H C = R^H R, one pass writes W <- (W - Q C) R^-1.  Four passes
//      over the basis per S steps instead of 2 S;
//   3. the S new Hessenberg columns follow from the change of basis:
//      A [q_k, Q_new(0:S-1)] = (R_all T - [H_old C''; 0]) Rhat^-1, with T the
//      (S+1) x S bidiagonal of the shifts, R_all the block's coefficients on
//      the whole basis, C'' their part on q_0..q_{k-1}; then the Givens
//      rotations, residual estimates and stop decisions of those S columns.
//
// The shifts are the Leja-ordered Ritz values of the first restart cycle, which
// runs the delayed CGS2 step (cg_api.cu).  A block whose Cholesky fails (the
// Newton basis lost rank numerically) ends the cycle at the columns already
// finished, so the solve restarts from the true residual instead of breaking.
// Numbers, layout and reductions follow the rest of the library: the basis is
// q_j normalised at V + j n, FP64 (or FP32 in mixed precision) complex,
// reductions in fixed order (two-level over blocks, as cg_dcgs2.cu).
#include <vector>

#include "cg_common.cuh"
#include "cg_internal.h"

namespace cg {

static constexpr int SS_THREADS = 256;
static constexpr int SS_WARPS = SS_THREADS / 32;
static constexpr int SS_CHUNK = 64;  // basis vectors per shared-memory chunk
// points per lane of the tile-major passes: the S block vectors of a tile stay
// in registers (at most 32 complex values per lane)
template <int S> constexpr int ss_u64() { return 32 / S > 8 ? 8 : (32 / S > 1 ? 32 / S : 1); }
template <int S> constexpr int ss_u32() { return 32 / S > 8 ? 8 : (32 / S > 1 ? 32 / S : 1); }
// the update pass keeps S x U accumulators next to the basis tiles: 4 FP64
// points per lane at S = 4 so that two blocks fit per SM (measured faster than
// 8 points with one block: 5.3 against 4.8 TB/s), while the dot pass is faster
// with 8 points and one block of 8 warps (4.9 against 4.0 TB/s)
template <int S> constexpr int ss_u64_upd() { return 16 / S > 4 ? 4 : (16 / S > 1 ? 16 / S : 1); }
template <typename CV> constexpr int ss_minb() { return sizeof(CV) == 16 ? 1 : 2; }
// stages of a warp's private basis-tile ring in the dot pass (cp.async, one
// commit group per basis vector, each lane copying and reading its own points)
static constexpr int SS_NST = 4;
// An FP64 block whose first pass keeps more than this fraction of every
// vector's squared norm skips the second pass: the first pass then leaves the
// block orthogonal to about eps / fraction (2e-15).  Measured: the 1024^2
// GMRES(100) blocks keep 0.1 to 0.3, and the 64^2 solves keep their step counts
// (699, 699, 673 with S = 2, 4, 8), which a 1e-2 threshold did not (711 with S = 2).
// Complex64 blocks always take both passes (eps = 6e-8).
static constexpr double SS_ONE_PASS = 0.1;

static __device__ __forceinline__ void cp_async_cv(double2 *dst, const double2 *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
static __device__ __forceinline__ void cp_async_cv(float2 *dst, const float2 *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
static __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> static __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// offsets (in double2) of the s-step scratch arrays in kp.ss; M1 = mcap + 1
struct SsLayout {
    long long C, Ct, Bc, G, Rt, Ai, Th, Mh, Sk, Ph, end;
    __host__ __device__ explicit SsLayout(int mcap) {
        const long long M1 = mcap + 1;
        C = 0;
        Ct = C + M1 * SS_MAX;
        Bc = Ct + M1 * SS_MAX;
        G = Bc + M1 * SS_MAX;
        Rt = G + SS_MAX * SS_MAX;
        Ai = Rt + SS_MAX * SS_MAX;
        Th = Ai + SS_MAX * SS_MAX;
        Mh = Th + SS_MAX;                        // [(mcap + SS_MAX + 1) * SS_MAX] work rows of k_ss_hess
        Sk = Mh + (M1 + SS_MAX) * SS_MAX;        // [M1] per block of the cycle: .x = 1 if its second pass was skipped
        Ph = Sk + M1;                            // [M1][SS_MAX] rows of H_old C'' from k_ss_hprod (long cycles)
        end = Ph + M1 * SS_MAX;
    }
};

long long sstep_scratch_elems(int mcap) { return SsLayout(mcap).end; }

// Which blocks of the last s-step cycle skipped their second pass (flags[b] for
// the block starting at column b S, nblocks of them); synchronises the stream.
int sstep_skipped(const KrylovPtrs &kp, int nblocks, std::vector<int> &flags, cudaStream_t s) {
    const SsLayout L(kp.mcap);
    std::vector<double2> h((size_t)nblocks);
    flags.assign((size_t)nblocks, 0);
    if (nblocks <= 0) return 0;
    if (int e = (int)cudaMemcpyAsync(h.data(), kp.ss + L.Sk, sizeof(double2) * h.size(), cudaMemcpyDeviceToHost, s))
        return e;
    if (int e = (int)cudaStreamSynchronize(s)) return e;
    for (int b = 0; b < nblocks; b++) flags[b] = h[b].x != 0.0;
    return 0;
}
static __host__ __device__ __forceinline__ int ss_pld(int mcap) { return 2 * SS_MAX * (mcap + 1) + 2 * SS_MAX * SS_MAX; }
int sstep_part_ld(int mcap) { return ss_pld(mcap); }

static __device__ __forceinline__ bool ss_last_of(unsigned int *ticket, unsigned int count) {
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

// Warp sum of V values (V a power of two, at most 32) by a reduce-scatter
// butterfly (V - 1 shuffles, then the remaining full-reduction rounds): on
// return lane L holds the total of value scatter_index<V>(L); fixed order.
template <int V> __device__ __forceinline__ int scatter_index(int lane) {
    int idx = 0;
#pragma unroll
    for (int off = 16, cnt = V; cnt > 1; off >>= 1, cnt >>= 1) idx = 2 * idx + ((lane & off) ? 1 : 0);
    return idx;
}
template <int V> __device__ __forceinline__ double warp_sum_scatter(double (&v)[V], int lane) {
    static_assert(V >= 1 && V <= 32 && (V & (V - 1)) == 0, "power of two");
    int off = 16;
#pragma unroll
    for (int cnt = V; cnt > 1; cnt >>= 1, off >>= 1) {
        const bool upper = (lane & off) != 0;
#pragma unroll
        for (int i = 0; i < cnt / 2; i++) {
            const double send = upper ? v[i] : v[i + cnt / 2];
            const double keep = upper ? v[i + cnt / 2] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    double t = v[0];
    for (; off >= 1; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    return t;
}
// lanes that write a scattered total: one per value index
template <int V> __device__ __forceinline__ bool scatter_writer(int lane) { return (lane & ((32 / V) - 1)) == 0; }

// ------------------------------------------------------------ Cholesky
// One block of SS_THREADS threads (the last block of the dot pass, once C and
// G are summed): Gp = G - C^H C (S x S), Gp = R^H R, A = R^-1, B = C R^-1, and
// the running totals Ct = Ct + C Rt, Rt = R Rt (Rt = I, Ct = 0 before pass 0).
// A failed factorisation (a pivot not above 1e-26 of the block's scale, or
// not finite) in the second pass ends the cycle at the columns already
// finished; in the first pass the block is projected without normalisation
// (R = I) and the second pass factors it.
template <int S> __device__ __forceinline__ void ss_chol(const KrylovPtrs &kp, int pass, double tau) {
    DevState *st = kp.st;
    const int k = st->k;
    const int nq = k + 1;
    const SsLayout L(kp.mcap);
    const double2 *C = kp.ss + L.C;
    double2 *Ct = kp.ss + L.Ct;
    double2 *Bc = kp.ss + L.Bc;
    const double2 *G = kp.ss + L.G;
    double2 *Rt = kp.ss + L.Rt;
    double2 *Ai = kp.ss + L.Ai;
    __shared__ double2 gp[S][S];
    __shared__ double2 rr[S][S];
    __shared__ double2 ai[S][S];
    __shared__ double2 rt_old[S][S];
    __shared__ double red[SS_WARPS][2];
    __shared__ int ok;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // C^H C, one entry per warp round: sum over the nq rows
    for (int e = 0; e < S * S; e++) {
        const int i = e / S, l = e % S;
        if (l < i) continue;
        double sr = 0.0, si = 0.0;
        for (int j = tid; j < nq; j += SS_THREADS) {
            const double2 a = C[j * SS_MAX + i], b = C[j * SS_MAX + l];
            sr += a.x * b.x + a.y * b.y;
            si += a.x * b.y - a.y * b.x;
        }
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (lane == 0) red[warp][0] = sr, red[warp][1] = si;
        __syncthreads();
        if (tid == 0) {
            double tr = 0.0, ti = 0.0;
            for (int w = 0; w < SS_WARPS; w++) tr += red[w][0], ti += red[w][1];
            const double2 g = G[i * SS_MAX + l];
            gp[i][l] = make_double2(g.x - tr, g.y - ti);
        }
        __syncthreads();
    }
    if (tid == 0) {
        for (int i = 0; i < S; i++)
            for (int l = 0; l < i; l++) gp[i][l] = cconj(gp[l][i]);
        double scale = 0.0;
        for (int i = 0; i < S; i++) scale = fmax(scale, G[i * SS_MAX + i].x);
        int good = isfinite(scale) && scale > 0.0;
        // Cholesky gp = R^H R (R upper), row by row
        for (int i = 0; i < S && good; i++) {
            double d = gp[i][i].x;
            for (int p = 0; p < i; p++) d -= rr[p][i].x * rr[p][i].x + rr[p][i].y * rr[p][i].y;
            if (!(d > 1e-26 * scale) || !isfinite(d)) {
                good = 0;
                break;
            }
            const double rii = sqrt(d);
            rr[i][i] = make_double2(rii, 0.0);
            for (int l = i + 1; l < S; l++) {
                double2 v = gp[i][l];
                for (int p = 0; p < i; p++) v = csub(v, cmul(cconj(rr[p][i]), rr[p][l]));
                rr[i][l] = make_double2(v.x / rii, v.y / rii);
            }
            for (int l = 0; l < i; l++) rr[i][l] = make_double2(0.0, 0.0);
        }
        int fallback = 0;
        if (!good && pass == 0 && isfinite(scale) && scale > 0.0) {
            // The Pythagorean update G - C^H C cancelled: the block lies almost in
            // the basis.  Take R = I for this pass, so that its update only projects
            // (W <- W - Q C) and the second pass factors the Gram matrix of the
            // projected block, where nothing cancels; the running totals come out
            // as Ct = C1 + C2, Rt = R2.  Non-finite coefficients still end the cycle.
            bool fin = true;
            for (int i = 0; i < S; i++)
                for (int l = 0; l < S; l++) fin = fin && isfinite(gp[i][l].x) && isfinite(gp[i][l].y);
            if (fin) {
                for (int i = 0; i < S; i++)
                    for (int l = 0; l < S; l++) rr[i][l] = make_double2(i == l ? 1.0 : 0.0, 0.0);
                good = 1;
                fallback = 1;
            }
        }
        if (pass == 0) {
            // One pass is enough when the projection cancelled little: the lost
            // orthogonality of a Pythagorean Cholesky pass is about eps * G_ii / R_ii^2
            // (the squared ratio of a block vector's norm to what stays of it after
            // projection and after the block's earlier vectors); when every
            // R_ii^2 / G_ii exceeds tau the second pass is skipped.
            double q = (good && !fallback) ? 1e300 : 0.0;
            for (int i = 0; i < S && good && !fallback; i++) q = fmin(q, (rr[i][i].x * rr[i][i].x) / G[i * SS_MAX + i].x);
            st->ss_one = q > tau ? 1 : 0;
            kp.ss[L.Sk + k / S] = make_double2((double)st->ss_one, 0.0);  // for the byte count of the profile
        }
        if (good) {
            // A = R^-1 (upper), column by column
            for (int l = 0; l < S; l++) {
                for (int i = S - 1; i >= 0; i--) {
                    double2 v = make_double2(i == l ? 1.0 : 0.0, 0.0);
                    for (int p = i + 1; p < S; p++) v = csub(v, cmul(rr[i][p], ai[p][l]));
                    const double inv = 1.0 / rr[i][i].x;
                    ai[i][l] = make_double2(v.x * inv, v.y * inv);
                }
            }
            for (int i = 0; i < S; i++)
                for (int l = 0; l < S; l++) {
                    rt_old[i][l] = pass == 0 ? make_double2(i == l ? 1.0 : 0.0, 0.0) : Rt[i * SS_MAX + l];
                    Ai[i * SS_MAX + l] = ai[i][l];
                }
        }
        ok = good;
    }
    __syncthreads();
    if (!ok) {
        if (tid == 0) {
            // end the cycle with the finished columns; none finished: no progress possible
            if (k == 0) st->brk = 1;
            st->stop = 1;
        }
        return;
    }
    // B = C R^-1 and Ct += C Rt_old (rows j = 0..k)
    for (int e = tid; e < nq * S; e += SS_THREADS) {
        const int j = e / S, l = e % S;
        double2 b = make_double2(0.0, 0.0), c = make_double2(0.0, 0.0);
        for (int i = 0; i < S; i++) {
            const double2 cji = C[j * SS_MAX + i];
            b = cadd(b, cmul(cji, ai[i][l]));
            c = cadd(c, cmul(cji, rt_old[i][l]));
        }
        Bc[j * SS_MAX + l] = b;
        Ct[j * SS_MAX + l] = pass == 0 ? c : cadd(Ct[j * SS_MAX + l], c);
    }
    if (tid < S * S) {
        const int i = tid / S, l = tid % S;
        double2 v = make_double2(0.0, 0.0);
        for (int p = 0; p < S; p++) v = cadd(v, cmul(rr[i][p], rt_old[p][l]));
        Rt[i * SS_MAX + l] = v;
    }
}

// ------------------------------------------------------------ block dots
// C[j][i] = <q_j, w_i> (j = 0..k, i < S), G[i][l] = <w_i, w_l>; tile-major:
// every warp keeps its tile of the S block vectors in registers and streams
// the basis over it.  Per-block partial rows part[b][2 S (k+1) + 2 S S] are
// summed in two fixed-order levels (groups of 16 blocks, then the groups).
// On short vectors the grid's second dimension splits the basis: slice y of
// gridDim.y takes the chunks of SS_CHUNK vectors with index = y mod gridDim.y
// and writes zeros in its rows for the others; the Gram matrix comes from
// slice 0.  (256^2: 256 tiles keep 32 blocks busy, each streaming the whole
// basis; four slices give 128.)
template <typename CV, int S, int U>
__global__ void __launch_bounds__(SS_THREADS, ss_minb<CV>()) k_ss_dots(const CV *__restrict__ V, long long n, KrylovPtrs kp,
                                                                       int pass) {
    typedef typename real_of<CV>::type R;
    DevState *st = kp.st;
    if (st->stop || (pass == 1 && st->ss_one)) return;
    const int k = st->k;
    const int nq = k + 1;
    const CV *W = V + (long long)(k + 1) * n;
    const int pld = ss_pld(kp.mcap);
    // [SS_WARPS][SS_CHUNK][2 S] and [SS_WARPS][2 S S] doubles, then the rings [SS_WARPS][SS_NST][U][32]
    extern __shared__ __align__(16) double sacc[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *my = sacc + (size_t)warp * SS_CHUNK * 2 * S;
    double *myg = sacc + (size_t)SS_WARPS * SS_CHUNK * 2 * S + (size_t)warp * 2 * S * S;
    CV *ring = reinterpret_cast<CV *>(sacc + (size_t)SS_WARPS * SS_CHUNK * 2 * S + (size_t)SS_WARPS * 2 * S * S) +
               (size_t)warp * SS_NST * U * 32;
    const long long TILE = 32LL * U;
    const long long ntile = (n + TILE - 1) / TILE;
    const long long nw = (long long)gridDim.x * SS_WARPS;
    for (int q = lane; q < 2 * S * S; q += 32) myg[q] = 0.0;
    const int bflat = blockIdx.y * gridDim.x + blockIdx.x;
    double *part = kp.part + (size_t)bflat * pld;
    bool gram_done = blockIdx.y != 0;
    for (int jc = 0; jc < nq; jc += SS_CHUNK) {
        const int nj = nq - jc < SS_CHUNK ? nq - jc : SS_CHUNK;
        if ((int)((jc / SS_CHUNK) % gridDim.y) != (int)blockIdx.y) {
            // another slice's chunk (block-uniform): this block adds nothing to it
            for (int q = threadIdx.x; q < nj * 2 * S; q += blockDim.x) part[2 * S * jc + q] = 0.0;
            continue;
        }
        for (int q = lane; q < nj * 2 * S; q += 32) my[q] = 0.0;
        __syncwarp();
        for (long long tile = (long long)blockIdx.x * SS_WARPS + warp; tile < ntile; tile += nw) {
            const long long e0 = tile * TILE + lane;
            const bool full = tile * TILE + TILE <= n;
            CV w[S][U];
#pragma unroll
            for (int i = 0; i < S; i++)
#pragma unroll
                for (int t = 0; t < U; t++) {
                    const long long e = e0 + 32 * t;
                    w[i][t] = (full || e < n) ? W[(long long)i * n + e] : czero<CV>();
                }
            if (!gram_done) {
                // Gram matrix of the block from the registers (upper triangle, once per tile)
#pragma unroll
                for (int i = 0; i < S; i++)
#pragma unroll
                    for (int l = i; l < S; l++) {
                        R gr = 0, gi = 0;
#pragma unroll
                        for (int t = 0; t < U; t++) {
                            gr = fma_r(w[i][t].y, w[l][t].y, fma_r(w[i][t].x, w[l][t].x, gr));
                            gi = fma_r(-w[i][t].y, w[l][t].x, fma_r(w[i][t].x, w[l][t].y, gi));
                        }
                        const double sr = warp_sum((double)gr), si = warp_sum((double)gi);
                        if (lane == 0) {
                            myg[2 * (i * S + l)] += sr;
                            myg[2 * (i * S + l) + 1] += si;
                        }
                    }
            }
            // basis tiles stream through the warp's ring, SS_NST - 1 vectors ahead
            auto issue = [&](int jj) {
                if (jj < nj) {
                    const CV *q = V + (long long)(jc + jj) * n;
                    CV *slot = ring + (size_t)(jj % SS_NST) * U * 32;
#pragma unroll
                    for (int t = 0; t < U; t++) {
                        const long long e = e0 + 32 * t;
                        if (full || e < n) cp_async_cv(slot + t * 32 + lane, q + e);
                    }
                }
                cp_async_commit();
            };
#pragma unroll
            for (int jj = 0; jj < SS_NST - 1; jj++) issue(jj);
            for (int j = 0; j < nj; j++) {
                issue(j + SS_NST - 1);
                cp_async_wait<SS_NST - 1>();  // this lane's copies of vector j have landed
                CV a[U];
                const CV *slot = ring + (size_t)(j % SS_NST) * U * 32;
#pragma unroll
                for (int t = 0; t < U; t++) {
                    const long long e = e0 + 32 * t;
                    a[t] = (full || e < n) ? slot[t * 32 + lane] : czero<CV>();
                }
                double d[2 * S];
#pragma unroll
                for (int i = 0; i < S; i++) {
                    R sr = 0, si = 0;
#pragma unroll
                    for (int t = 0; t < U; t++) {
                        // conj(q) w, four FMAs per point
                        sr = fma_r(a[t].y, w[i][t].y, fma_r(a[t].x, w[i][t].x, sr));
                        si = fma_r(-a[t].y, w[i][t].x, fma_r(a[t].x, w[i][t].y, si));
                    }
                    d[2 * i] = (double)sr;
                    d[2 * i + 1] = (double)si;
                }
                const double tot = warp_sum_scatter<2 * S>(d, lane);
                if (scatter_writer<2 * S>(lane)) my[2 * S * j + scatter_index<2 * S>(lane)] += tot;
            }
        }
        gram_done = true;
        __syncthreads();
        for (int q = threadIdx.x; q < nj * 2 * S; q += blockDim.x) {
            double t = 0.0;
            for (int wq = 0; wq < SS_WARPS; wq++) t += sacc[(size_t)wq * SS_CHUNK * 2 * S + q];
            part[2 * S * jc + q] = t;
        }
        __syncthreads();
    }
    for (int q = threadIdx.x; q < 2 * S * S; q += blockDim.x) {
        double t = 0.0;
        for (int wq = 0; wq < SS_WARPS; wq++) t += sacc[(size_t)SS_WARPS * SS_CHUNK * 2 * S + (size_t)wq * 2 * S * S + q];
        part[2 * S * nq + q] = t;
    }
    // two-level fixed-order sum of the block rows
    const int nvals = 2 * S * nq + 2 * S * S;
    const int nb = gridDim.x * gridDim.y, ng = (nb + 15) / 16;
    const int g = bflat / 16;
    const int gsz = nb - g * 16 < 16 ? nb - g * 16 : 16;
    if (!ss_last_of(&kp.tickets[g], (unsigned int)gsz)) return;
    for (int q = threadIdx.x; q < nvals; q += blockDim.x) {
        double s = 0.0;
        for (int b = g * 16; b < g * 16 + gsz; b++) s += __ldcg(kp.part + (size_t)b * pld + q);
        kp.gpart[(size_t)g * pld + q] = s;
    }
    if (!ss_last_of(&st->counter[5], (unsigned int)ng)) return;
    const SsLayout L(kp.mcap);
    double *C = reinterpret_cast<double *>(kp.ss + L.C);
    double *G = reinterpret_cast<double *>(kp.ss + L.G);
    for (int q = threadIdx.x; q < nvals; q += blockDim.x) {
        double s = 0.0;
        for (int gg = 0; gg < ng; gg++) s += __ldcg(kp.gpart + (size_t)gg * pld + q);
        if (q < 2 * S * nq) {
            const int j = q / (2 * S), i = (q / 2) % S;
            C[2 * (j * SS_MAX + i) + (q & 1)] = s;
        } else {
            const int r = q - 2 * S * nq;
            const int i = (r / 2) / S, l = (r / 2) % S;
            G[2 * (i * SS_MAX + l) + (r & 1)] = s;
        }
    }
    // the last block goes on with the pass's Cholesky (C and G are complete)
    __syncthreads();
    ss_chol<S>(kp, pass, sizeof(CV) == 16 ? SS_ONE_PASS : 2.0);  // q <= 1: complex64 never skips
}

// ------------------------------------------------------------ update
// W <- W A - Q B in place (A = R^-1 of the pass, B = C R^-1); tile-major.
template <typename CV, int S, int U>
__global__ void __launch_bounds__(SS_THREADS, 2) k_ss_update(CV *__restrict__ V, long long n, KrylovPtrs kp, int pass) {
    typedef typename real_of<CV>::type R;
    DevState *st = kp.st;
    if (st->stop || (pass == 1 && st->ss_one)) return;
    const int k = st->k;
    const int nq = k + 1;
    CV *W = V + (long long)(k + 1) * n;
    const SsLayout L(kp.mcap);
    __shared__ CV sa[S][S];
    __shared__ CV sb[SS_CHUNK][S];
    for (int e = threadIdx.x; e < S * S; e += blockDim.x) {
        const double2 a = kp.ss[L.Ai + (e / S) * SS_MAX + (e % S)];
        sa[e / S][e % S] = mk<CV>((R)a.x, (R)a.y);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    extern __shared__ __align__(16) unsigned char ss_upd_smem[];  // rings [SS_WARPS][SS_NST][U][32]
    CV *ring = reinterpret_cast<CV *>(ss_upd_smem) + (size_t)warp * SS_NST * U * 32;
    const long long TILE = 32LL * U;
    const long long ntile = (n + TILE - 1) / TILE;
    const long long nw = (long long)gridDim.x * SS_WARPS;
    // the coefficient chunks are shared by every tile of the block, so each
    // tile is visited once per chunk; the partial outputs stay in registers
    // only within one tile, hence the loop order tile -> chunk with the
    // chunk reloaded per tile (the coefficients are tiny next to the basis)
    for (long long tile0 = (long long)blockIdx.x * SS_WARPS; tile0 < ntile; tile0 += nw) {
        const long long tile = tile0 + warp;
        const bool live = tile < ntile;
        const long long e0 = tile * TILE + lane;
        const bool full = live && tile * TILE + TILE <= n;
        // FP64: -Q B first, W A last, so the block vectors (read one at a time at
        // the end) are never live next to the accumulators and the basis tiles;
        // FP32 (twice the points per lane fit): W A first, then -Q B
        constexpr bool WA_LAST = sizeof(CV) == 16;
        CV acc[S][U];
#pragma unroll
        for (int l = 0; l < S; l++)
#pragma unroll
            for (int t = 0; t < U; t++) acc[l][t] = czero<CV>();
        // the coefficients in sa are written before the first tile: a barrier
        // before W A is read (the chunk loop below has its own for W A last)
        if (!WA_LAST) __syncthreads();
        if (!WA_LAST && live) {
#pragma unroll
            for (int i = 0; i < S; i++) {
                CV w[U];
#pragma unroll
                for (int t = 0; t < U; t++) {
                    const long long e = e0 + 32 * t;
                    w[t] = (full || e < n) ? W[(long long)i * n + e] : czero<CV>();
                }
#pragma unroll
                for (int l = i; l < S; l++)
#pragma unroll
                    for (int t = 0; t < U; t++) acc[l][t] = cfma(acc[l][t], w[t], sa[i][l]);
            }
        }
        for (int jc = 0; jc < nq; jc += SS_CHUNK) {
            const int nj = nq - jc < SS_CHUNK ? nq - jc : SS_CHUNK;
            __syncthreads();
            for (int e = threadIdx.x; e < nj * S; e += blockDim.x) {
                const double2 b = kp.ss[L.Bc + (long long)(jc + e / S) * SS_MAX + (e % S)];
                sb[e / S][e % S] = mk<CV>((R)b.x, (R)b.y);
            }
            __syncthreads();
            if (live) {
                // basis tiles stream through the warp's ring, SS_NST - 1 vectors ahead
                auto issue = [&](int jj) {
                    if (jj < nj) {
                        const CV *q = V + (long long)(jc + jj) * n;
                        CV *slot = ring + (size_t)(jj % SS_NST) * U * 32;
#pragma unroll
                        for (int t = 0; t < U; t++) {
                            const long long e = e0 + 32 * t;
                            if (full || e < n) cp_async_cv(slot + t * 32 + lane, q + e);
                        }
                    }
                    cp_async_commit();
                };
#pragma unroll
                for (int jj = 0; jj < SS_NST - 1; jj++) issue(jj);
                for (int j = 0; j < nj; j++) {
                    issue(j + SS_NST - 1);
                    cp_async_wait<SS_NST - 1>();  // this lane's copies of vector j have landed
                    CV a[U];
                    const CV *slot = ring + (size_t)(j % SS_NST) * U * 32;
#pragma unroll
                    for (int t = 0; t < U; t++) {
                        const long long e = e0 + 32 * t;
                        a[t] = (full || e < n) ? slot[t * 32 + lane] : czero<CV>();
                    }
#pragma unroll
                    for (int l = 0; l < S; l++) {
                        const CV b = sb[j][l];
#pragma unroll
                        for (int t = 0; t < U; t++) acc[l][t] = cfms(acc[l][t], a[t], b);
                    }
                }
            }
        }
        if (WA_LAST && live) {
#pragma unroll
            for (int i = 0; i < S; i++) {
                CV w[U];
#pragma unroll
                for (int t = 0; t < U; t++) {
                    const long long e = e0 + 32 * t;
                    w[t] = (full || e < n) ? W[(long long)i * n + e] : czero<CV>();
                }
#pragma unroll
                for (int l = i; l < S; l++)
#pragma unroll
                    for (int t = 0; t < U; t++) acc[l][t] = cfma(acc[l][t], w[t], sa[i][l]);
            }
        }
        if (live) {
            __syncwarp();
#pragma unroll
            for (int l = 0; l < S; l++)
#pragma unroll
                for (int t = 0; t < U; t++) {
                    const long long e = e0 + 32 * t;
                    if (full || e < n) W[(long long)l * n + e] = acc[l][t];
                }
        }
    }
}

// ------------------------------------------------------------ Hessenberg + Givens
// Row r of H_old C'' (r = 0..k): sum over the columns l = max(r-1, 0)..k-1 of
// the upper Hessenberg H_old of H[r][l] Ct[l][j], j < S - 1, lanes strided over
// l and a fixed-order warp sum.  Shared by the one-block Hessenberg kernel and
// the many-block product that long cycles launch before it (the same sum in
// the same order, so both give the same bits).
template <int S>
__device__ __forceinline__ void ss_hrow(const KrylovPtrs &kp, const double2 *Ct, int r, int k, int ld, int lane,
                                        double (&hs)[2 * (S - 1) > 0 ? 2 * (S - 1) : 1]) {
#pragma unroll
    for (int q = 0; q < 2 * (S - 1); q++) hs[q] = 0.0;
    for (int l = (r > 0 ? r - 1 : 0) + lane; l < k; l += 32) {
        const double2 hv = kp.Hm[(size_t)r * ld + l];
#pragma unroll
        for (int jj = 0; jj < S - 1; jj++) {
            const double2 p = cmul(hv, Ct[l * SS_MAX + jj]);
            hs[2 * jj] += p.x;
            hs[2 * jj + 1] += p.y;
        }
    }
#pragma unroll
    for (int q = 0; q < 2 * (S - 1); q++) hs[q] = warp_sum(hs[q]);
}

// H_old C'' over many blocks, one warp per row, into the Ph rows: at a basis of
// k vectors the product reads k^2 / 2 entries of H (128 MB at k = 4000), which
// one block of threads would stream at a single SM's bandwidth.
template <int S> __global__ void __launch_bounds__(SS_THREADS) k_ss_hprod(KrylovPtrs kp) {
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k;
    const int ld = kp.mcap + 1;
    const SsLayout L(kp.mcap);
    const double2 *Ct = kp.ss + L.Ct;
    double2 *P = kp.ss + L.Ph;
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * SS_WARPS;
    for (int r = blockIdx.x * SS_WARPS + (threadIdx.x >> 5); r <= k; r += nw) {
        double hs[2 * (S - 1) > 0 ? 2 * (S - 1) : 1];
        ss_hrow<S>(kp, Ct, r, k, ld, lane, hs);
#pragma unroll
        for (int jj = 0; jj < S - 1; jj++)
            if (lane == jj) P[(size_t)r * SS_MAX + jj] = make_double2(hs[2 * jj], hs[2 * jj + 1]);
    }
}

// One block: the S new columns k..k+S-1 of H (rows 0..k+S) from the block's
// coefficients (Ct, Rt), the shifts and the earlier columns of H, then their
// Givens rotations, residual estimates and the stop decision.  p_ready: the
// rows of H_old C'' are in Ph (k_ss_hprod ran first).
template <int S> __global__ void __launch_bounds__(SS_THREADS) k_ss_hess(KrylovPtrs kp, int m_in_smem, int p_ready) {
    DevState *st = kp.st;
    if (st->stop) return;
    const int k = st->k;
    const int ld = kp.mcap + 1;
    const SsLayout L(kp.mcap);
    const double2 *Ct = kp.ss + L.Ct;
    const double2 *Rt = kp.ss + L.Rt;
    const double2 *Th = kp.ss + L.Th;
    const int tid = threadIdx.x;
    // work rows [(k + S + 1) * S], row-major: in shared memory when the launch
    // provides (mcap + SS_MAX + 1) * S of them, else in the global scratch (long cycles)
    extern __shared__ double2 ss_hess_smem[];
    double2 *M = m_in_smem ? ss_hess_smem : kp.ss + L.Mh;
    __shared__ double2 rh[S][S];  // Rhat
    const int nr = k + S + 1;
    // Rall[r][c], c = 0..S: column 0 = e_k; column c >= 1: Ct(:, c-1) on rows <= k, Rt(:, c-1) below
    auto rall = [&](int r, int c) -> double2 {
        if (c == 0) return make_double2(r == k ? 1.0 : 0.0, 0.0);
        if (r <= k) return Ct[r * SS_MAX + (c - 1)];
        const int i = r - k - 1;
        return i <= c - 1 ? Rt[i * SS_MAX + (c - 1)] : make_double2(0.0, 0.0);
    };
    // M = Rall T - [H_old C''; 0]: one warp per row r, its lanes over the
    // columns l of H_old (upper Hessenberg: l >= r - 1), fixed-order warp sums
    const int warp = tid >> 5, lane = tid & 31;
    const double2 *P = kp.ss + L.Ph;
    for (int r = warp; r < nr; r += SS_WARPS) {
        double hs[2 * (S - 1) > 0 ? 2 * (S - 1) : 1];
#pragma unroll
        for (int q = 0; q < 2 * (S - 1); q++) hs[q] = 0.0;
        if (r <= k) {
            if (p_ready) {
#pragma unroll
                for (int jj = 0; jj < S - 1; jj++) {
                    const double2 pv = P[(size_t)r * SS_MAX + jj];
                    hs[2 * jj] = pv.x;
                    hs[2 * jj + 1] = pv.y;
                }
            } else {
                ss_hrow<S>(kp, Ct, r, k, ld, lane, hs);
            }
        }
#pragma unroll
        for (int j = 0; j < S; j++)
            if (lane == j) {
                double2 v = cadd(cmul(rall(r, j), Th[j]), rall(r, j + 1));
                if (r <= k && j >= 1) v = csub(v, make_double2(hs[2 * (j - 1)], hs[2 * (j - 1) + 1]));
                M[r * S + j] = v;
            }
    }
    if (tid < S * S) {
        const int r = tid / S, c = tid % S;
        rh[r][c] = rall(k + r, c);
    }
    __syncthreads();
    // H_new = M Rhat^-1: per row, forward substitution over the columns
    for (int r = tid; r < nr; r += SS_THREADS) {
        double2 hrow[S];
#pragma unroll
        for (int c = 0; c < S; c++) {
            double2 v = M[r * S + c];
#pragma unroll
            for (int p = 0; p < c; p++) v = csub(v, cmul(hrow[p], rh[p][c]));
            const double2 d = rh[c][c];
            const double dd = d.x * d.x + d.y * d.y;
            hrow[c] = cscale(cmulc(d, v), 1.0 / dd);  // v / d
        }
#pragma unroll
        for (int c = 0; c < S; c++) M[r * S + c] = hrow[c];
    }
    __syncthreads();
    // columns inside the restart length (a last block may reach past it)
    const int cols = st->m - k < S ? st->m - k : S;
    // store the Hessenberg part of the new columns (rows <= k + c + 1)
    for (int e = tid; e < nr * S; e += SS_THREADS) {
        const int r = e / S, c = e % S;
        if (c < cols && r <= k + c + 1) kp.Hm[(size_t)r * ld + (k + c)] = M[e];
    }
    // the earlier rotations applied to each new column (one thread per column)
    if (tid < cols) {
        const int c = tid;
        double2 carry = M[0 * S + c];
        // the loads do not depend on the carry: fetch 8 rotations ahead of the chain
        constexpr int RC = 8;
        for (int j0 = 0; j0 < k; j0 += RC) {
            double2 cj[RC], nx[RC];
            double sj[RC];
#pragma unroll
            for (int u = 0; u < RC; u++)
                if (j0 + u < k) {
                    cj[u] = kp.cs[j0 + u];
                    sj[u] = kp.sn[j0 + u];
                    nx[u] = M[(j0 + u + 1) * S + c];
                }
#pragma unroll
            for (int u = 0; u < RC; u++)
                if (j0 + u < k) {
                    kp.Rm[(size_t)(k + c) * ld + j0 + u] = cadd(cmul(cconj(cj[u]), carry), cscale(nx[u], sj[u]));
                    carry = csub(cmul(cj[u], nx[u]), cscale(carry, sj[u]));
                }
        }
        M[k * S + c] = carry;
    }
    __syncthreads();
    if (tid != 0) return;
    // the block's own rotations, column by column
    int it = st->it, stop = 0, done = 0;
    for (int c = 0; c < cols && !stop; c++) {
        const int col = k + c;
        // rotations k..col-1 (made in this block) on the rest of column col
        double2 carry = M[k * S + c];
        for (int j = k; j < col; j++) {
            const double2 cj = kp.cs[j];
            const double sj = kp.sn[j];
            const double2 nx = M[(j + 1) * S + c];
            kp.Rm[(size_t)col * ld + j] = cadd(cmul(cconj(cj), carry), cscale(nx, sj));
            carry = csub(cmul(cj, nx), cscale(carry, sj));
        }
        // H(col+1, col) = Rt(c, c) / Rhat(c, c) is real and positive by construction
        const double hk1 = M[(col + 1) * S + c].x;
        const double rho = hypot(hypot(carry.x, carry.y), hk1);
        double2 cs;
        double sn;
        if (!(rho > 0.0) || !isfinite(rho)) {
            cs = make_double2(1.0, 0.0);
            sn = 0.0;
        } else {
            cs = make_double2(carry.x / rho, carry.y / rho);
            sn = hk1 / rho;
        }
        kp.Rm[(size_t)col * ld + col] = cadd(cmul(cconj(cs), carry), make_double2(sn * hk1, 0.0));
        kp.cs[col] = cs;
        kp.sn[col] = sn;
        const double2 gk = kp.g[col];
        kp.g[col + 1] = cscale(gk, -sn);
        kp.g[col] = cmul(cconj(cs), gk);
        it++;
        const double gabs = hypot(gk.x, gk.y) * sn;
        const double est = gabs / st->nb;
        st->est = est;
        kp.hist[it] = est;
        done = c + 1;
        if (!isfinite(est)) {
            st->status = 4;
            stop = 1;
        }
        if (gabs <= st->tol * st->nb || gabs <= st->inner_tol * st->beta0) stop = 1;
        if (col + 1 >= st->m) stop = 1;
        if (it >= st->maxit) stop = 1;
        if (!(hk1 > 1e-300)) stop = 1;  // the Krylov space is invariant: exact in it
    }
    st->it = it;
    st->ncol = k + done;
    st->k = k + done;
    st->stop = stop;
}

// q_0 = r / ||r|| at the start of an s-step cycle (k_cycle_begin leaves r in V_0)
template <typename CV> __global__ void k_ss_norm0(CV *__restrict__ V, long long n, KrylovPtrs kp) {
    DevState *st = kp.st;
    if (st->stop) return;
    typedef typename real_of<CV>::type R;
    const R inv = (R)(1.0 / st->beta0);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        V[e] = cscale(V[e], inv);
}

// ------------------------------------------------------------ launchers
template <typename K> static int ss_smem(K kern, size_t bytes) {
    return smem_optin(kern, bytes);
}

static constexpr int SS_U32 = 8;  // tile width used to size the grid

// Grid of a tile-major pass: the fewest rounds of warp tiles the resident
// blocks allow (`per_sm` blocks of SS_WARPS warps on each of `sms` SMs), then
// the fewest blocks that still finish in that many rounds, so every warp gets
// the same number of tiles (1024^2 FP64 dots: 4096 tiles -> 128 blocks of 4
// rounds, where 148 resident blocks would leave the fourth round 46 % full);
// at most `cap` blocks (the rows of the partial buffers).
static int ss_grid(long long ntile, int sms, int per_sm, int cap) {
    const long long resident = (long long)sms * per_sm * SS_WARPS;
    const long long rounds = (ntile + resident - 1) / resident;
    long long g = (ntile + rounds * SS_WARPS - 1) / (rounds * SS_WARPS);
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

// Basis slices of the dot pass (its grid's second dimension): as many as fill
// `per_sm` blocks on every SM next to the `nblk` blocks that the tiles keep
// busy, at most 8, within the partial rows of the buffer.
static int ss_slices(int nblk, int sms, int per_sm, int rows) {
    int y = (sms * per_sm) / nblk;
    if (y > 8) y = 8;
    while (y > 1 && (long long)y * nblk > rows) y--;
    return y < 1 ? 1 : y;
}

template <int S> static int ss_dots_t(int prec, const void *V, long long n, const KrylovPtrs &kp, int sms, int pass,
                                      cudaStream_t s) {
    const size_t acc = sizeof(double) * ((size_t)SS_WARPS * SS_CHUNK * 2 * S + (size_t)SS_WARPS * 2 * S * S);
    const int cap = sstep_blocks(sms, n);
    const int rows = sstep_part_rows(sms);
    if (prec == 0) {
        constexpr int U = ss_u64<S>();
        const size_t smem = acc + sizeof(double2) * (size_t)SS_WARPS * SS_NST * U * 32;
        auto kern = k_ss_dots<double2, S, U>;
        if (int e = ss_smem(kern, smem)) return e;
        const int nblk = ss_grid((n + 32 * U - 1) / (32 * U), sms, ss_minb<double2>(), cap);
        const dim3 grid(nblk, ss_slices(nblk, sms, ss_minb<double2>(), rows));
        kern<<<grid, SS_THREADS, smem, s>>>((const double2 *)V, n, kp, pass);
    } else {
        constexpr int U = ss_u32<S>();
        const size_t smem = acc + sizeof(float2) * (size_t)SS_WARPS * SS_NST * U * 32;
        auto kern = k_ss_dots<float2, S, U>;
        if (int e = ss_smem(kern, smem)) return e;
        const int nblk = ss_grid((n + 32 * U - 1) / (32 * U), sms, ss_minb<float2>(), cap);
        const dim3 grid(nblk, ss_slices(nblk, sms, ss_minb<float2>(), rows));
        kern<<<grid, SS_THREADS, smem, s>>>((const float2 *)V, n, kp, pass);
    }
    return (int)cudaGetLastError();
}

template <int S> static int ss_update_t(int prec, void *V, long long n, const KrylovPtrs &kp, int sms, int pass,
                                        cudaStream_t s) {
    const int cap = 2 * sms;  // the update writes no partial rows: the cap is occupancy only
    if (prec == 0) {
        constexpr int U = ss_u64_upd<S>();
        const size_t smem = sizeof(double2) * (size_t)SS_WARPS * SS_NST * U * 32;
        auto kern = k_ss_update<double2, S, U>;
        if (int e = ss_smem(kern, smem)) return e;
        kern<<<ss_grid((n + 32 * U - 1) / (32 * U), sms, 2, cap), SS_THREADS, smem, s>>>((double2 *)V, n, kp, pass);
    } else {
        constexpr int U = ss_u32<S>();
        const size_t smem = sizeof(float2) * (size_t)SS_WARPS * SS_NST * U * 32;
        auto kern = k_ss_update<float2, S, U>;
        if (int e = ss_smem(kern, smem)) return e;
        kern<<<ss_grid((n + 32 * U - 1) / (32 * U), sms, 2, cap), SS_THREADS, smem, s>>>((float2 *)V, n, kp, pass);
    }
    return (int)cudaGetLastError();
}

// Blocks from this basis size on get the many-block H_old C'' first: below it
// the one-block product costs less than the extra launch (restart-100 cycles
// never reach it).
static constexpr int SS_HPROD_MIN = 512;

template <int S> static int ss_hess_t(const KrylovPtrs &kp, int k, cudaStream_t s) {
    const size_t smem = sizeof(double2) * (size_t)(kp.mcap + SS_MAX + 1) * S;
    const bool in_smem = smem <= 48 * 1024;
    const bool many = k >= SS_HPROD_MIN;
    if (many) {
        int g = (k + 1 + SS_WARPS - 1) / SS_WARPS;  // one warp per row
        if (g > 1184) g = 1184;
        k_ss_hprod<S><<<g, SS_THREADS, 0, s>>>(kp);
    }
    if (in_smem)
        if (int e = smem_optin(k_ss_hess<S>, smem)) return e;
    k_ss_hess<S><<<1, SS_THREADS, in_smem ? smem : 0, s>>>(kp, in_smem ? 1 : 0, many ? 1 : 0);
    return (int)cudaGetLastError();
}

#define SS_DISPATCH(S, CALL)                  \
    switch (S) {                              \
        case 2: return CALL(2);               \
        case 4: return CALL(4);               \
        case 8: return CALL(8);               \
        default: return -1;                   \
    }

int sstep_supported(int S) { return S == 2 || S == 4 || S == 8; }

int sstep_part_rows(int sms) { return 2 * sms; }

int sstep_blocks(int sms, long long n) {
    const long long tiles = (n + 32 * SS_U32 - 1) / (32 * SS_U32);
    long long g = 2LL * sms;
    const long long cap = (tiles + SS_WARPS - 1) / SS_WARPS;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

int launch_ss_dots(int prec, const void *V, long long n, const KrylovPtrs &kp, int S, int sms, int pass,
                   cudaStream_t s) {
#define CALL(S_) ss_dots_t<S_>(prec, V, n, kp, sms, pass, s)
    SS_DISPATCH(S, CALL)
#undef CALL
}

int launch_ss_update(int prec, void *V, long long n, const KrylovPtrs &kp, int S, int sms, int pass, cudaStream_t s) {
#define CALL(S_) ss_update_t<S_>(prec, V, n, kp, sms, pass, s)
    SS_DISPATCH(S, CALL)
#undef CALL
}

int launch_ss_hess(const KrylovPtrs &kp, int S, int k, cudaStream_t s) {
#define CALL(S_) ss_hess_t<S_>(kp, k, s)
    SS_DISPATCH(S, CALL)
#undef CALL
}

int launch_ss_norm0(int prec, void *V, long long n, const KrylovPtrs &kp, cudaStream_t s) {
    const int nb = (int)((n + 255) / 256 > 1024 ? 1024 : (n + 255) / 256);
    if (prec == 0) k_ss_norm0<double2><<<nb, 256, 0, s>>>((double2 *)V, n, kp);
    else k_ss_norm0<float2><<<nb, 256, 0, s>>>((float2 *)V, n, kp);
    return (int)cudaGetLastError();
}

}  // namespace cg
