// Stockham radix-16 / radix-8 FFT building blocks for the circulant-embedding matvec.
//
// The reference applies its BTTB operator with two cuFFT calls on an odd
// (2N-1)^2 grid plus three elementwise kernels (CUDA_GMRES/Fast_matvec.cuh:1-28).
// Here the embedding is a power-of-two L x L grid (L >= 2N-1, normally L = 2N)
// and the 1D transforms are the project's own: a Stockham auto-sort FFT
// (formulation of Govindaraju, Lloyd, Dotsenko, Smith and Manferdelli,
// "High performance discrete Fourier transforms on graphics processors", SC08)
// where each thread owns E = 16 (or 8) points:
//
//   stage s with radix R and span Ns reads  a[j + r L/R]          (r < R)
//   multiplies by the twiddle  w_{Ns R}^{(j mod Ns) r} = w_L^{(j mod Ns) r L/(Ns R)},
//   does an R-point DFT and writes b[(j/Ns) Ns R + (j mod Ns) + q Ns] (q < R).
//
// Twiddles come from per-stage tables (see Plan::twoff): stage s >= 1 keeps
// w_{Ns R}^{k r} for k < Ns, 1 <= r < R at twoff(s) + (r-1) Ns + k, so the
// threads of a warp (consecutive k) read consecutive entries instead of
// entries k r L/(Ns R) apart in one length-L table.
//
// Thread t of a transform owns butterflies j = t + b*TPR (TPR = L/E threads).
// The first stage (span 1, no twiddles) reads and the last stage (span L/R)
// writes the "canonical" register set reg[p] = element t + p*TPR, so a
// transform can start from coalesced global loads and end in coalesced global
// stores or in the next transform without touching shared memory.  Middle
// stages exchange through shared memory padded by one element every 16, which
// keeps the 16-byte accesses of a quarter warp on distinct banks.
#pragma once

#include "cg_common.cuh"

namespace cg {

// ------------------------------------------------------------ small DFTs
// In-place natural-order DFTs on register arrays.  INV selects the sign of
// the exponent: forward exp(-2 pi i k/R), inverse exp(+2 pi i k/R), unscaled.

// multiply by w_4^1 = -i (forward) or +i (inverse)
template <bool INV, typename C> __device__ __forceinline__ C mul_w4(C a) {
    return INV ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
}
// multiply by w_8^1 = (1 -/+ i)/sqrt(2)
template <bool INV, typename C> __device__ __forceinline__ C mul_w8_1(C a) {
    typedef typename real_of<C>::type R;
    const R h = (R)0.70710678118654752440;
    return INV ? mk<C>((a.x - a.y) * h, (a.x + a.y) * h) : mk<C>((a.x + a.y) * h, (a.y - a.x) * h);
}
// multiply by w_8^3 = (-1 -/+ i)/sqrt(2)
template <bool INV, typename C> __device__ __forceinline__ C mul_w8_3(C a) {
    typedef typename real_of<C>::type R;
    const R h = (R)0.70710678118654752440;
    return INV ? mk<C>(-(a.x + a.y) * h, (a.x - a.y) * h) : mk<C>((a.y - a.x) * h, -(a.x + a.y) * h);
}
// multiply by (cr + i*ci) with ci negated for the forward direction
template <bool INV, typename C>
__device__ __forceinline__ C mul_cs(C a, typename real_of<C>::type cr, typename real_of<C>::type si) {
    typedef typename real_of<C>::type R;
    const R ci = INV ? si : -si;
    return mk<C>(a.x * cr - a.y * ci, a.x * ci + a.y * cr);
}

template <bool INV, typename C> __device__ __forceinline__ void dft2(C *v) {
    C t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
}

template <bool INV, typename C> __device__ __forceinline__ void dft4(C *v) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = mul_w4<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}

// combine two half-length DFTs: X[k] = E[k] + w^k O[k], X[k+h] = E[k] - w^k O[k]
template <bool INV, typename C> __device__ __forceinline__ void dft8(C *v) {
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    dft4<INV>(e);
    dft4<INV>(o);
    o[1] = mul_w8_1<INV>(o[1]);
    o[2] = mul_w4<INV>(o[2]);
    o[3] = mul_w8_3<INV>(o[3]);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[k] = cadd(e[k], o[k]);
        v[k + 4] = csub(e[k], o[k]);
    }
}

// cos(k pi/8), sin(k pi/8) for k = 1, 3 (exact decimal expansions of the
// mathematical constants, rounded by the compiler)
#define CG_C1 0.92387953251128675613
#define CG_S1 0.38268343236508977173

template <bool INV, typename C> __device__ __forceinline__ C mul_w16(C a, int k) {
    typedef typename real_of<C>::type R;
    switch (k) {
        case 1: return mul_cs<INV>(a, (R)CG_C1, (R)CG_S1);
        case 2: return mul_w8_1<INV>(a);
        case 3: return mul_cs<INV>(a, (R)CG_S1, (R)CG_C1);
        case 4: return mul_w4<INV>(a);
        case 5: return mul_cs<INV>(a, -(R)CG_S1, (R)CG_C1);
        case 6: return mul_w8_3<INV>(a);
        case 7: return mul_cs<INV>(a, -(R)CG_C1, (R)CG_S1);
        default: return a;
    }
}

template <bool INV, typename C> __device__ __forceinline__ void dft16(C *v) {
    C e[8], o[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
        e[r] = v[2 * r];
        o[r] = v[2 * r + 1];
    }
    dft8<INV>(e);
    dft8<INV>(o);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        C t = mul_w16<INV>(o[k], k);
        v[k] = cadd(e[k], t);
        v[k + 8] = csub(e[k], t);
    }
}

template <int R, bool INV, typename C> __device__ __forceinline__ void dft(C *v) {
    if constexpr (R == 2) dft2<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else if constexpr (R == 16) dft16<INV>(v);
}

// DFT of length R whose inputs R/2 .. R-1 are zero (the zero-padded half of
// the embedding): X[2m] = DFT_{R/2}(v)[m], X[2m+1] = DFT_{R/2}(v[r] w_R^r)[m].
template <int R, bool INV, typename C> __device__ __forceinline__ void dft_half_input(C *v) {
    if constexpr (R == 2) {
        v[1] = v[0];
    } else {
    C a[R / 2], b[R / 2];
#pragma unroll
    for (int r = 0; r < R / 2; r++) a[r] = v[r];
    if constexpr (R == 16) {
#pragma unroll
        for (int r = 0; r < 8; r++) b[r] = mul_w16<INV>(v[r], r);
    } else if constexpr (R == 8) {
        b[0] = v[0];
        b[1] = mul_w8_1<INV>(v[1]);
        b[2] = mul_w4<INV>(v[2]);
        b[3] = mul_w8_3<INV>(v[3]);
    } else {  // R == 4
        b[0] = v[0];
        b[1] = mul_w4<INV>(v[1]);
    }
    dft<R / 2, INV>(a);
    dft<R / 2, INV>(b);
#pragma unroll
    for (int m = 0; m < R / 2; m++) {
        v[2 * m] = a[m];
        v[2 * m + 1] = b[m];
    }
    }
}

// ------------------------------------------------------------ plans
// Length L = E^a * rem with E points per thread (16 or 8): stages of radix E,
// then one stage of radix rem < E.  Lengths below E use one stage of radix L.
template <int L, int E0 = 16> struct Plan {
    static constexpr int E = (L >= E0) ? E0 : L;
    static constexpr int TPR = L / E;
    __host__ __device__ static constexpr int ilog(int v) { return v <= 1 ? 0 : 1 + ilog(v / 2); }
    static constexpr int LOG = ilog(L);
    static constexpr int LOGE = ilog(E);
    static constexpr int NFULL = LOG / LOGE;
    static constexpr int REM = 1 << (LOG - NFULL * LOGE);
    static constexpr int NST = NFULL + (REM > 1 ? 1 : 0);
    __host__ __device__ static constexpr int radix(int s) { return s < NFULL ? E : REM; }
    __host__ __device__ static constexpr int span(int s) { return s == 0 ? 1 : span(s - 1) * radix(s - 1); }
    // padded shared-memory index (one pad element every 16)
    static __device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
    static constexpr int SMEM_ELEMS = L + L / 16;
    // offset of stage s's twiddles (s >= 1); the tables of all stages take
    // sum_s (R_s - 1) Ns_s = L - R_0 < L entries
    __host__ __device__ static constexpr int twoff(int s) {
        return s <= 1 ? 0 : twoff(s - 1) + (radix(s - 1) - 1) * span(s - 1);
    }
};

// Twiddle tables of one precision, 4 L entries: [E0 = 16 forward | E0 = 16
// inverse | E0 = 8 forward | E0 = 8 inverse], each in the per-stage layout of
// Plan<L, E0> (forward exp(-2 pi i m / L), inverse the conjugates).
template <int L, int E0, bool INV, typename C> __device__ __forceinline__ const C *tw_table(const C *tw) {
    return tw + (E0 == 16 ? 0 : 2 * L) + (INV ? L : 0);
}

// Exponent m of entry i of the per-stage table of a length-L transform with
// E0 points per thread (the entry is exp(-/+ 2 pi i m / L)), or -1 for the
// unused entries i >= L - R_0.  Mirrors Plan at run time, for the host and
// for device-side table builders.
__host__ __device__ inline int twiddle_exponent(int L, int E0, int i) {
    const int E = L >= E0 ? E0 : L;
    int lg = 0, lge = 0;
    while ((1 << lg) < L) lg++;
    while ((1 << lge) < E) lge++;
    const int nfull = lg / lge, rem = 1 << (lg - nfull * lge);
    const int nst = nfull + (rem > 1 ? 1 : 0);
    int ns = 1, off = 0;
    for (int st = 0; st < nst; st++) {
        const int R = st < nfull ? E : rem;
        if (st > 0) {
            const int size = (R - 1) * ns;
            if (i < off + size) {
                const int r = (i - off) / ns + 1, k = (i - off) % ns;
                return k * r * (L / (ns * R));
            }
            off += size;
        }
        ns *= R;
    }
    return -1;
}

// Barrier of the threads that share one transform: the whole block (NT = 0)
// or the NT threads of named barrier `id` (1..15; NT a multiple of 32), so
// that several transforms in one block do not wait on each other.
template <int NT> __device__ __forceinline__ void fft_barrier(int id) {
    if constexpr (NT == 0) {
        __syncthreads();
    } else {
        static_assert(NT % 32 == 0, "named barriers count whole warps");
        asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(NT) : "memory");
    }
}

// Twiddles w^{k r}, r = 1..R-1, of one butterfly (w = w_{Ns R}), from its two
// base values w^k and (R >= 8) w^{4k}: the other powers are products of at
// most three factors, so each carries a few units of rounding more than a
// table entry (well inside the transform's own error), while the table reads
// -- the largest share of a pass's L1/L2 load traffic when every power was
// read -- drop from R-1 to 2.  CONJ: the conjugate powers (the inverse
// transform from the forward table's bases).  w[0] is unused.
template <int R, bool CONJ, typename C> __device__ __forceinline__ void stage_twiddles(C w1, C w4, C (&w)[R]) {
    if constexpr (CONJ) {
        w1 = cconj(w1);
        w4 = cconj(w4);
    }
    w[0] = mk<C>(1, 0);
    w[1] = w1;
    if constexpr (R == 4) {
        w[2] = cmul(w[1], w[1]);
        w[3] = cmul(w[2], w[1]);
    } else if constexpr (R >= 8) {
        w[4] = w4;
        w[2] = cmul(w[1], w[1]);
        w[3] = cmul(w[2], w[1]);
        w[5] = cmul(w[4], w[1]);
        w[6] = cmul(w[4], w[2]);
        w[7] = cmul(w[4], w[3]);
        if constexpr (R == 16) {
            w[8] = cmul(w[4], w[4]);
            w[12] = cmul(w[8], w[4]);
#pragma unroll
            for (int r = 1; r < 4; r++) {
                w[8 + r] = cmul(w[8], w[r]);
                w[12 + r] = cmul(w[12], w[r]);
            }
        }
    }
}

// Base twiddles of every butterfly a thread runs in stages 1.. of a length-L
// transform (stage 0 has none): per butterfly w^k and, for radix >= 8, w^{4k}
// (table entries r = 1 and r = 4 of the stage's [r][k] layout).  They depend
// only on the thread, so kernels that run many transforms (the persistent
// column passes) load them once and keep them in registers.
template <int L, int E0> struct TwBase {
    typedef Plan<L, E0> P;
    __host__ __device__ static constexpr int per(int s) {
        return s == 0 ? 0 : (P::E / P::radix(s)) * (P::radix(s) >= 8 ? 2 : 1);
    }
    __host__ __device__ static constexpr int off(int s) { return s <= 1 ? 0 : off(s - 1) + per(s - 1); }
    __host__ __device__ static constexpr int total() { return P::NST <= 1 ? 0 : off(P::NST - 1) + per(P::NST - 1); }
    static constexpr int COUNT = total() > 0 ? total() : 1;
};

template <int L, int E0, int S> struct TwBaseLoad {
    typedef Plan<L, E0> P;
    template <typename C>
    static __device__ __forceinline__ void run(const C *__restrict__ tw, int t, C (&wb)[TwBase<L, E0>::COUNT]) {
        if constexpr (S < P::NST) {
            constexpr int R = P::radix(S), Ns = P::span(S), NB = P::E / R, O = TwBase<L, E0>::off(S);
#pragma unroll
            for (int b = 0; b < NB; b++) {
                const int k = (t + b * P::TPR) % Ns;
                const C *__restrict__ ts = tw + P::twoff(S) + k;
                if constexpr (R >= 8) {
                    wb[O + 2 * b] = __ldg(ts);
                    wb[O + 2 * b + 1] = __ldg(ts + 3 * Ns);
                } else {
                    wb[O + b] = __ldg(ts);
                }
            }
            TwBaseLoad<L, E0, S + 1>::run(tw, t, wb);
        }
    }
};

// Loads this thread's base twiddles from the table set `tw` (the forward
// table of the E0 plan).
template <int L, int E0, typename C>
__device__ __forceinline__ void load_tw_base(const C *__restrict__ tw, int t, C (&wb)[TwBase<L, E0>::COUNT]) {
    TwBaseLoad<L, E0, 1>::run(tw_table<L, E0, false>(tw), t, wb);
}

// One Stockham stage S of a length-L transform (compile-time radix and span).
// tmp holds the previous stage's butterfly outputs (tmp[b*Rp + q]) on entry
// and this stage's outputs on exit; the last stage stores canonical reg.
template <int L, int E0, bool INV, bool HALF_IN, int S, int SMS, int NT = 0, bool CONJ = false> struct Stage {
    typedef Plan<L, E0> P;
    static constexpr int E = P::E;
    static constexpr int TPR = P::TPR;
    static constexpr int R = P::radix(S);
    static constexpr int Ns = P::span(S);
    static constexpr int NB = E / R;  // butterflies per thread in this stage
    template <typename C>
    static __device__ __forceinline__ void run(C (&reg)[E], C (&tmp)[E], C *sm, const C (&wb)[TwBase<L, E0>::COUNT],
                                               int t, int bar) {
        if constexpr (S > 0) {
            // write the previous stage's outputs, then read this stage's inputs
            constexpr int Rp = P::radix(S - 1);
            constexpr int Nsp = P::span(S - 1);
            constexpr int NBp = E / Rp;
            fft_barrier<NT>(bar);
#pragma unroll
            for (int b = 0; b < NBp; b++) {
                const int j = t + b * TPR;
                const int base = (j / Nsp) * Nsp * Rp + (j % Nsp);
#pragma unroll
                for (int q = 0; q < Rp; q++) sm[P::pad(base + q * Nsp) * SMS] = tmp[b * Rp + q];
            }
            fft_barrier<NT>(bar);
#pragma unroll
            for (int b = 0; b < NB; b++) {
                const int j = t + b * TPR;
                constexpr int O = TwBase<L, E0>::off(S);
                C w[R];
                if constexpr (R >= 8) stage_twiddles<R, CONJ>(wb[O + 2 * b], wb[O + 2 * b + 1], w);
                else stage_twiddles<R, CONJ>(wb[O + b], wb[O + b], w);
#pragma unroll
                for (int r = 0; r < R; r++) {
                    C v = sm[P::pad(j + r * (L / R)) * SMS];
                    if (r > 0) v = cmul(v, w[r]);
                    tmp[b * R + r] = v;
                }
            }
        } else {
#pragma unroll
            for (int b = 0; b < NB; b++)
#pragma unroll
                for (int r = 0; r < R; r++) tmp[b * R + r] = reg[b + r * NB];
        }
#pragma unroll
        for (int b = 0; b < NB; b++) {
            if constexpr (S == 0 && HALF_IN) dft_half_input<R, INV>(tmp + b * R);
            else dft<R, INV>(tmp + b * R);
        }
        if constexpr (S == P::NST - 1) {
#pragma unroll
            for (int b = 0; b < NB; b++)
#pragma unroll
                for (int q = 0; q < R; q++) reg[b + q * NB] = tmp[b * R + q];
        } else {
            Stage<L, E0, INV, HALF_IN, S + 1, SMS, NT, CONJ>::run(reg, tmp, sm, wb, t, bar);
        }
    }
};

// Runs one length-L transform owned by TPR threads (this thread is t).
// reg[p] holds element t + p*TPR on entry and on exit.  sm is this
// transform's padded shared-memory region: element i lives at sm[pad(i) * SMS]
// (SMS > 1 interleaves the regions of SMS transforms element by element, which
// keeps the column kernels' accesses on distinct banks).
// HALF_IN: inputs L/2 .. L-1 are zero (first stage uses dft_half_input).
// Every thread of the block (NT = 0), or of named barrier `bar` (NT threads),
// must call this the same number of times (it contains barriers).  tw is the
// base of the 4 L-entry table set (tw_table picks the plan's and direction's table).
// The stage twiddles' base values are loaded at the start (all stages at
// once, so their latency overlaps the first stage), from the direction's own
// table.
template <int L, int E0, bool INV, bool HALF_IN, int SMS = 1, int NT = 0, typename C>
__device__ __forceinline__ void fft_run(C (&reg)[Plan<L, E0>::E], C *sm, const C *__restrict__ tw, int t,
                                        int bar = 0) {
    C tmp[Plan<L, E0>::E];
    C wb[TwBase<L, E0>::COUNT];
    TwBaseLoad<L, E0, 1>::run(tw_table<L, E0, INV>(tw), t, wb);
    Stage<L, E0, INV, HALF_IN, 0, SMS, NT>::run(reg, tmp, sm, wb, t, bar);
}

// Same with base twiddles the caller loaded once (load_tw_base, forward
// table); the inverse uses their conjugates.
template <int L, int E0, bool INV, bool HALF_IN, int SMS = 1, int NT = 0, typename C>
__device__ __forceinline__ void fft_run_wb(C (&reg)[Plan<L, E0>::E], C *sm, const C (&wb)[TwBase<L, E0>::COUNT],
                                           int t, int bar = 0) {
    C tmp[Plan<L, E0>::E];
    Stage<L, E0, INV, HALF_IN, 0, SMS, NT, INV>::run(reg, tmp, sm, wb, t, bar);
}

}  // namespace cg
