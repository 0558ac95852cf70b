// Internal declarations shared by the cugmres translation units (not part of
// the C-ABI; the public interface is include/cugmres.h).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <vector>

struct cg_ctx;  // solver context (cg_api.cu)

namespace cg {

// Opt `kern` in to `dyn` bytes of dynamic shared memory when its static shared
// memory and `dyn` together pass the 48 KB that a launch may use without
// opting in.  Comparing `dyn` alone let kernels with static arrays fail to
// launch just below the threshold (the delayed-CGS2 step kernel, 6.4 KB
// static, at restarts of about 1070 to 1230).
template <typename K> inline int smem_optin(K kern, size_t dyn) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, kern);
    if (e != cudaSuccess) return (int)e;
    if (a.sharedSizeBytes + dyn <= 48 * 1024) return 0;
    return (int)cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
}

// Solver state kept in device memory so that no host synchronisation is
// needed per Arnoldi step (the reference copies Jtotal(i+1,0) to the host and
// the residual back every iteration, CUDA_GMRES/GMRES.cuh:369-371).
struct DevState {
    int k;         // Arnoldi column being built in this cycle (basis holds k+1 vectors)
    int it;        // iterations completed over all cycles
    int stop;      // 1: the current cycle takes no further Arnoldi step
    int status;    // 0 running, 1 converged, 2 iteration budget spent, 3 breakdown, 4 non-finite
    int m;         // restart length of the current cycle
    int maxit;     // total iteration budget
    int rotation;  // 0 unitary Givens, 1 the reference's formula
    int fixed;     // 1: never stop on the residual estimate (reference semantics)
    int cycles;    // cycles started
    int brk;       // breakdown seen in this cycle
    int ncol;      // Hessenberg columns finalised in this cycle
    int ortho;     // 0 delayed CGS2, 1 CGS2
    double tol;       // relative tolerance on ||b - A x|| / ||b||
    double inner_tol; // cycle stops when |g_{k+1}| <= inner_tol * beta0 (mixed precision)
    double nb;        // ||b||
    double beta0;     // ||r|| at the start of the current cycle
    double est;       // last relative residual estimate |g_{k+1}| / ||b||
    double true_res;  // last true relative residual ||b - A x|| / ||b||
    double wnorm2;    // ||w||^2 of the vector just orthogonalised
    double scalar;    // scratch scalar result of a norm reduction
    double cu, cw;    // delayed CGS2 axpy scalars: q_k = cu u - sum P_j q_j,
    double2 du;       //   u_{k+1} = cw w + du u - sum S_j q_j
    double2 delta;    // q_k^H w of the current delayed CGS2 step
    unsigned int counter[8];  // tickets of the last-block reductions
    int ss_one;               // s-step: the block's first Gram-Schmidt pass was enough (second pass skipped)
};

// Device workspace of one Krylov cycle (restart m, budget maxit).
struct KrylovPtrs {
    DevState *st;
    double *scale;   // [m+2] lazy normalisation of the stored basis vectors
    double2 *h1;     // [m+1] first Gram-Schmidt coefficients
    double2 *h2;     // [m+1] reorthogonalisation coefficients
    double2 *Rm;     // [(m+1) * m] triangular factor, column k at Rm + k*(m+1)
    double2 *cs;     // [m] rotation cosines (complex)
    double *sn;      // [m] rotation sines (real)
    double2 *g;      // [m+1] rotated right-hand side
    double2 *y;      // [m] least-squares solution
    double *hist;    // [maxit+1] relative residual history
    double *part;    // [nblk_dot * (m+1) * 2] dot partials
    double *npart;   // [nblk_max] norm partials
    double2 *Hm;     // [(m+1) * (m+1)] unrotated Hessenberg, row-major: H(i,j) at Hm[i*(m+1) + j]
    double2 *D1;     // [m+2] <q_j, u_k> (j < k) and <u_k, u_k> (j = k)
    double2 *D2;     // [m+2] <q_j, w> (j < k) and <u_k, w> (j = k)
    double2 *tv;     // [m+2] first-pass coefficients of A q_{k-1}
    double2 *P;      // [m+1] axpy coefficients for q_k
    double2 *S;      // [m+1] axpy coefficients for u_{k+1}
    double *gpart;   // [ceil(nblk_dots2 / 16) * 4 * part_ld] group sums of the dot partials
    unsigned int *tickets;  // [ceil(nblk_dots2 / 16)] arrival counters of those groups (reset by the last)
    double2 *ss = nullptr;  // s-step scratch (cg_sstep.cu: block coefficients, Gram, shifts, work rows)
    int mcap;        // allocated restart capacity (leading dimension of Rm / part)
    // Bucket of systems solved in lockstep (one launch covers all of them,
    // system = blockIdx.y): every array above (st included) of system s lies
    // s * sys_ws bytes after system 0's, and its basis s * sys_v elements after
    // V.  A single solve has nsys = 1 and zero strides.
    long long sys_ws = 0;
    long long sys_v = 0;
    int nsys = 1;
};

// This block's system of a bucket: kp with every workspace pointer moved to
// system blockIdx.y (no change for a single solve).
__device__ __forceinline__ KrylovPtrs kp_sys(KrylovPtrs kp) {
    if (kp.sys_ws == 0) return kp;
    const long long o = (long long)blockIdx.y * kp.sys_ws;
#define CG_MOVE(f) kp.f = kp.f ? reinterpret_cast<decltype(kp.f)>(reinterpret_cast<char *>(kp.f) + o) : kp.f
    CG_MOVE(st); CG_MOVE(scale); CG_MOVE(h1); CG_MOVE(h2); CG_MOVE(Rm); CG_MOVE(cs); CG_MOVE(sn);
    CG_MOVE(g); CG_MOVE(y); CG_MOVE(hist); CG_MOVE(part); CG_MOVE(npart); CG_MOVE(Hm); CG_MOVE(D1);
    CG_MOVE(D2); CG_MOVE(tv); CG_MOVE(P); CG_MOVE(S); CG_MOVE(gpart); CG_MOVE(tickets); CG_MOVE(ss);
#undef CG_MOVE
    return kp;
}
template <typename T> __device__ __forceinline__ T *sys_vec(T *V, const KrylovPtrs &kp) {
    return V + (long long)blockIdx.y * kp.sys_v;
}

// Matvec launch parameters for one precision (C = double2 or float2, R its real type).
struct MatvecArgs {
    int N, L;
    int vfwd, vcols, vinv;  // launch shape of each pass (0..matvec_variants(L)-1), chosen by the autotuner
    const void *gq;     // quarter spectrum (C)
    const void *cdiag;  // N x N real diagonal k0^2 chi (R)
    const void *tw;     // L twiddles (C)
    void *T;            // N x L intermediate (C)
    int transpose = 0;  // 1: A^T x = x - diag(c) G x (contrast applied after the convolution)
    int sms = 148;      // multiprocessors of the device (grid of the persistent column pass)
    int nsys = 1;       // systems of a bucket (grid.y of every pass)
    // per-system strides of a bucket: workspace bytes (DevState, scale and the
    // norm partials move with it), then elements of the contrast, of T, of the
    // quarter spectrum and of the right-hand side
    long long sys_ws = 0, sys_c = 0, sys_T = 0, sys_gq = 0, sys_b = 0;
};

// The per-system strides a matvec kernel needs (see MatvecArgs).
struct SysSel {
    long long ws, c, T, gq, b;
};
inline SysSel sys_sel(const MatvecArgs &a) { return SysSel{a.sys_ws, a.sys_c, a.sys_T, a.sys_gq, a.sys_b}; }
template <typename T> __device__ __forceinline__ T *sys_move_bytes(T *p, long long stride_bytes) {
    return p ? reinterpret_cast<T *>(reinterpret_cast<char *>(const_cast<void *>((const void *)p)) +
                                     (long long)blockIdx.y * stride_bytes)
             : p;
}

// Reference to a basis vector selected by the device-side Arnoldi index:
// ptr = base + (st ? st->k + koff : 0) * stride.
struct VecSel {
    void *base;
    long long stride;
    int koff;
    long long sys = 0;  // elements between the vectors of consecutive systems of a bucket
    int abs = 0;        // 1: vector koff itself; 0: vector st->k + koff (the cycle's current column)
};

// kernel launchers (cg_matvec.cu)
int launch_rows_forward(int prec, const MatvecArgs &a, VecSel x, const double *xscale_base, const DevState *st,
                        int gate, cudaStream_t s);
int launch_cols_convolve(int prec, const MatvecArgs &a, const DevState *st, int gate, cudaStream_t s);
// mode 0: y = s (1 - shift) x - conv = (A - shift) (s x);  mode 1: y = b - x + conv
// (y may be float2 while the matvec is double2: out_prec)
// Pass 3 of a matvec y = (A - shift) x fused with pass 1 of the next matvec on y
// (same precision, plain operator): y is stored and c y transformed into T.
int launch_rows_inv_fwd(int prec, const MatvecArgs &a, VecSel x, VecSel y, const DevState *st, int gate,
                        cudaStream_t s, double2 shift);
int launch_rows_inverse(int prec, int mode, int out_prec, const MatvecArgs &a, VecSel x, const double *xscale_base,
                        const void *b, VecSel y, double *npart, const DevState *st, int gate, cudaStream_t s,
                        double2 shift = double2{0.0, 0.0});
int rows_per_block(int variant, int L);
int fft_supported(int L);
int matvec_variants(int L);
// 1 if launch shape v runs the column pass as a persistent kernel (one block
// of about 200 KB shared memory on every SM)
int matvec_variant_persistent(int v);
// marks a context whose GPU is shared with other contexts' solves (set by the
// batch solver before its first operator)
void ctx_set_shared_gpu(cg_ctx *c, bool on);
// Device buffers of a context's current operator (FP64), read by the bucket
// solver, which copies each system's spectrum and contrast into its own arrays.
struct OpView {
    int N, L, sms;
    int var[2][3];  // launch shapes of the three matvec passes, FP64 and FP32
    const double2 *gq64;
    const float2 *gq32;
    const double *c64;
    const float *c32;
    const double2 *tw64;
    const float2 *tw32;
    cudaStream_t stream;
};
int ctx_op_view(const cg_ctx *c, OpView *v);

// full (unpruned) forward 2D transform of an L x L FP64 array, used to build the spectrum
int launch_fft2d_full_fp64(int L, double2 *a, const double2 *tw, cudaStream_t s);
// Green's-function block g[d1*N + d2] of `kind` (CG_GREEN_*) on the device.
int launch_green_block(int kind, int N, double k0, double h, double2 *out, int sms, cudaStream_t s);

// kernel launchers (cg_krylov.cu)
int launch_dots(int prec_v, const void *V, long long n, const KrylovPtrs &kp, VecSel w, double2 *out, int ctr,
                int nblk, int gate, cudaStream_t s);
int launch_axpy(int prec_v, int prec_w, const void *V, long long n, const KrylovPtrs &kp, const double2 *src,
                double sign, int nj_mode, VecSel w, int want_norm, int ctr, int nblk, int gate, cudaStream_t s);
int launch_givens(const KrylovPtrs &kp, cudaStream_t s);
// delayed CGS2 step (cg_dcgs2.cu)
int launch_dots2(int prec_v, const void *V, long long n, const KrylovPtrs &kp, int nblk, int sms, cudaStream_t s);
int launch_dcgs2_step(const KrylovPtrs &kp, cudaStream_t s);
int launch_axpy2(int prec_v, const void *V, long long n, const KrylovPtrs &kp, int nblk, int sms, cudaStream_t s);
int dots2_blocks(int prec_v, int sms, int mcap, long long n);
int axpy2_blocks(int prec_v, int sms, int mcap, long long n);
// partials per block of the two-RHS dot pass
__host__ __device__ inline int dots2_part_ld(int mcap) { return 2 * (mcap + 1) > 64 ? 2 * (mcap + 1) : 64; }
int launch_backsolve(const KrylovPtrs &kp, cudaStream_t s);
int launch_cycle_begin(const KrylovPtrs &kp, int nparts, cudaStream_t s);
// ortho 0: delayed CGS2, 1: CGS2, for the cycle k_cycle_begin has just set up
int launch_set_ortho(const KrylovPtrs &kp, int ortho, cudaStream_t s);
// s-step Arnoldi (cg_sstep.cu): S steps per block, S in {2, 4, 8}
constexpr int SS_MAX = 8;
int sstep_supported(int S);
long long sstep_scratch_elems(int mcap);  // double2 entries of KrylovPtrs::ss
int sstep_part_ld(int mcap);              // partials per block of the block dot pass
int sstep_blocks(int sms, long long n);   // grid of the block dot and update passes
int sstep_part_rows(int sms);              // partial rows of the dot pass, basis slices included
int sstep_skipped(const KrylovPtrs &kp, int nblocks, std::vector<int> &flags, cudaStream_t s);
int launch_ss_norm0(int prec, void *V, long long n, const KrylovPtrs &kp, cudaStream_t s);
// block dots of pass `pass` (0 or 1); the last block also runs the pass's Cholesky.
// The dot and update passes size their grids from the SM count (sms).
int launch_ss_dots(int prec, const void *V, long long n, const KrylovPtrs &kp, int S, int sms, int pass,
                   cudaStream_t s);
int launch_ss_update(int prec, void *V, long long n, const KrylovPtrs &kp, int S, int sms, int pass, cudaStream_t s);
// k: the basis size the block starts at (b S), which picks the many-block
// H_old C'' product for long cycles
int launch_ss_hess(const KrylovPtrs &kp, int S, int k, cudaStream_t s);
int launch_norm2(int prec, const void *v, long long n, double *npart, unsigned int *counter, double *out, int nblk,
                 cudaStream_t s);
int launch_convert(int from_prec, int to_prec, const void *src, void *dst, long long n, cudaStream_t s);

// gate codes for the per-iteration kernels
enum { GATE_NONE = 0, GATE_STOP = 1 };
// nj_mode for launch_axpy: number of basis vectors used
enum { NJ_K_PLUS_1 = 0, NJ_K = 1, NJ_NCOL = 2 };

}  // namespace cg
