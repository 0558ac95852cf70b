/* cugmres_b200 -- C-ABI of the B200 GMRES solver for A = I - G diag(c),
 * G a symmetric block-Toeplitz-Toeplitz-block (BTTB) Green's-function matrix
 * on an N x N grid and c a real diagonal (c = k0^2 chi for the Helmholtz
 * Lippmann-Schwinger / GFIEM system).
 *
 * Every function returns a status code (CG_OK = 0) and never exits the
 * process.  Arrays are row-major N x N grids of interleaved complex numbers
 * (re, im); pointers may be host or device memory (detected per call).
 * A context owns one CUDA stream and its device workspace; calls on one
 * context must not overlap, different contexts are independent.
 *
 * Reference interfaces each entry point replaces (paths inside the reference
 * project "Benchmarks of CUDA-based GMRES Solver for Toeplitz and Hankel
 * Matrices and Applications to Topology Optimization of Photonic Devices/"):
 *   CUDA_GMRES/GMRES.cuh:22-35           Fast_GMRES_with_CUDA   -> cugmres_solve, cugmres_fast_gmres
 *   CUDA_GMRES/Fast_matvec.cuh:1-28      G_x_fft_matvec (+ crop) -> cugmres_matvec
 *   CUDA_GMRES/launch_GMRES.cuh:93-142   cuFFT plan + FFT of G   -> cugmres_create, cugmres_set_operator
 *   MKL_GMRES_test_09122019/source/loop_functions.h:128-168
 *                                        Green_matrix_create_MKL -> cugmres_green_block
 *   PyGMRES/GMRES.py:47-57               matvec(x, eps, k)       -> cugmres_matvec (via cugmres_b200.matvec)
 */
#ifndef CUGMRES_H
#define CUGMRES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } cg_c128;
typedef struct { float re, im; } cg_c64;
typedef struct cg_ctx cg_ctx;

/* status codes */
enum {
    CG_OK = 0,
    CG_ERR_INVALID = 1,         /* bad argument (null pointer, size, option)            */
    CG_ERR_CUDA = 2,            /* a CUDA runtime call failed                           */
    CG_ERR_NOT_CONVERGED = 3,   /* iteration budget spent before reaching tol           */
    CG_ERR_BREAKDOWN = 4,       /* Arnoldi breakdown without convergence                */
    CG_ERR_NONFINITE = 5,       /* NaN or Inf met in the input or during the iteration  */
    CG_ERR_TIMEOUT = 6,         /* opts.timeout_s elapsed                               */
    CG_ERR_NOT_IMPLEMENTED = 7, /* size or mode the library does not support            */
    CG_ERR_NO_OPERATOR = 8,     /* cugmres_set_operator has not been called             */
    CG_ERR_OOM = 9              /* device allocation failed                             */
};

/* precision of the Krylov cycle */
enum {
    CG_PREC_FP64 = 0,  /* complex128 everywhere                                         */
    CG_PREC_MIXED = 1  /* complex64 Arnoldi cycles inside an FP64 residual/update loop  */
};

/* Givens rotation formula */
enum {
    CG_GIVENS_UNITARY = 0,   /* [[conj(c), s], [-s, c]]: true GMRES minimal residual          */
    CG_GIVENS_REFERENCE = 1  /* [[c, s], [-s, c]] with c = h_ii/rho as the reference writes it
                                (MKL_GMRES_test_09122019/source/loop_functions.h:630-689)      */
};

/* Arnoldi orthogonalisation */
enum {
    CG_ORTHO_DCGS2 = 0, /* classical Gram-Schmidt, reorthogonalisation delayed one step: 2 passes over the basis per step */
    CG_ORTHO_CGS2 = 1,  /* classical Gram-Schmidt with one immediate reorthogonalisation: 4 passes per step            */
    CG_ORTHO_SSTEP = 2  /* s-step: opts->sstep Arnoldi steps per block (a Newton basis of sstep matvecs, block
                           Gram-Schmidt with Pythagorean Cholesky, the second pass only where the first
                           cancelled): 2 to 4 passes over the basis per block; the Newton shifts are the Ritz
                           values of a 24-step CG_ORTHO_DCGS2 run from b made before the solve               */
};

/* Green's-function constructions for cugmres_green_block */
enum {
    CG_GREEN_HELMHOLTZ = 0, /* G(d) = (i/4) H0(k0 h |d|) h^2, self term (i pi a/(2k0)) H1(k0 a) - 1/k0^2, pi a^2 = h^2 */
    CG_GREEN_REFERENCE = 1, /* g(i,j) = (i/4) H0(k sqrt((i-1/2)^2 + j^2)) with k = 2*3.14f/(N/6.f), rounded to float
                               (loop_functions.h:128-168)                                            */
    CG_GREEN_PYGMRES = 2    /* g(i,j) = (i/4) H0(k0 sqrt(i^2 + (j-1/2)^2)) in double, the NumPy reference's
                               get_green_matrix(k0, N) (PyGMRES/GMRES.py:20-27); h is ignored        */
};

typedef struct {
    int restart;        /* Krylov dimension per cycle m (>= 1)                                 */
    int max_iter;       /* total Arnoldi steps allowed                                         */
    double tol;         /* stop when ||b - A x|| / ||b|| <= tol                                */
    int precision;      /* CG_PREC_*                                                           */
    int givens;         /* CG_GIVENS_*                                                         */
    double inner_tol;   /* mixed: a complex64 cycle ends when its residual dropped by this      */
    int zero_x0;        /* 1: ignore x on entry and start from 0                               */
    int fixed_iterations; /* 1: reference semantics -- one cycle of exactly max_iter steps,
                             tol is an absolute threshold on ||b - A x0|| only                 */
    double timeout_s;   /* <= 0: none; otherwise the solve returns CG_ERR_TIMEOUT after this    */
    int ortho;          /* CG_ORTHO_*                                                          */
    int preconditioner; /* CG_PRECOND_*; CG_PRECOND_LEARNED needs cugmres_set_preconditioner;
                           flexible GMRES: a preconditioned and a plain probe cycle, then every
                           cycle in the mode that last reduced the true residual faster per
                           second (plain for good once a preconditioned cycle fails to reduce
                           it); preconditioned cycles last at most 40 steps                 */
    int learned_x0;     /* 1: with a preconditioner attached and zero_x0, start from x0 = M(b)
                           (kept only if ||b - A x0|| < ||b||, otherwise x0 = 0)             */
    int transpose;      /* 1: solve A^T x = b, A^T = I - diag(c) G (the adjoint system of the
                           reference's gradient path, CUDA_GMRES/GMRES.cuh:97-111; the adjoint
                           A^H x = b is conj of the A^T solve with conj(b))                    */
    int sstep;          /* CG_ORTHO_SSTEP: steps per block, 2, 4 or 8 (0: 4); restart >= sstep      */
    int reserved[3];
} cg_opts;

/* right preconditioning */
enum {
    CG_PRECOND_NONE = 0,    /* plain GMRES                                                     */
    CG_PRECOND_LEARNED = 1  /* flexible GMRES with the attached spectral-convolution network:
                               the first cycle runs preconditioned, the second plain, then
                               each cycle uses the mode that cut the true residual faster
                               per second; a preconditioned cycle that does not reduce it
                               switches the rest of the solve to plain GMRES               */
};

typedef struct {
    int status;                   /* CG_OK, CG_ERR_NOT_CONVERGED, CG_ERR_BREAKDOWN, ...   */
    int iterations;               /* Arnoldi steps taken                                  */
    int cycles;                   /* restart cycles started                               */
    double rel_residual_estimate; /* last |g_{k+1}| / ||b||                               */
    double rel_residual_true;     /* ||b - A x|| / ||b|| of the returned x (FP64 matvec)  */
    double seconds;               /* wall time of the solve                               */
    int preconditioned_cycles;    /* cycles run with the learned preconditioner           */
    int x0_learned;               /* 1: the solve started from x0 = M(b)                  */
} cg_result;

const char *cugmres_strerror(int status);
int cugmres_version(void);
void cugmres_default_opts(cg_opts *opts);

/* Creates a context on `device` with its own non-blocking stream. */
int cugmres_create(cg_ctx **ctx, int device);
int cugmres_destroy(cg_ctx *ctx);
/* Optional: run on a caller-provided cudaStream_t instead of the context's own. */
int cugmres_set_stream(cg_ctx *ctx, void *stream);
int cugmres_synchronize(cg_ctx *ctx);

/* Host-side Green's-function block g[d1*N + d2], 0 <= d1, d2 < N, for the
 * symmetric BTTB matrix G(i1-i2, j1-j2) = g(|i1-i2|, |j1-j2|).  No GPU needed. */
int cugmres_green_block(int kind, int N, double k0, double h, cg_c128 *out);

/* Sets the operator A = I - G diag(chi_scale * chi).  g_block: N x N as
 * produced by cugmres_green_block (host or device), chi: N x N real.
 * Builds the L x L circulant spectrum (L = smallest power of two >= 2N-1) on
 * the GPU in FP64 and keeps FP64 and FP32 copies of its even quarter. */
int cugmres_set_operator(cg_ctx *ctx, int N, const cg_c128 *g_block, const double *chi, double chi_scale);
/* The whole set-up on the GPU: the Green's block of `kind` (CG_GREEN_*, same
 * formulas as cugmres_green_block, evaluated with CUDA's double-precision
 * Bessel functions), embedding and spectrum; only chi is read from the host. */
int cugmres_set_operator_green(cg_ctx *ctx, int kind, int N, double k0, double h, const double *chi,
                               double chi_scale);
/* The Green's block into device memory `out` (N*N cg_c128) on `stream`. */
int cugmres_green_block_device(int kind, int N, double k0, double h, cg_c128 *out, void *stream);
/* Same from the reference's spatial (2N-1) x (2N-1) circulant G_prep
 * (CUDA_GMRES/Release/input/G_prep_N.txt layout, row-major, complex64);
 * its first N x N block is the g_block. */
int cugmres_set_operator_circulant(cg_ctx *ctx, int N, const cg_c64 *g_prep, const double *chi, double chi_scale);
int cugmres_grid_size(const cg_ctx *ctx, int *N, int *L);
/* Launch shapes the autotuner chose for the three matvec passes (row forward,
 * column convolution, row inverse) of `precision`; shapes[3] receives indices
 * 0..9 (0 for embeddings L < 128).  Tuning runs in cugmres_set_operator and is
 * cached per device in $CUGMRES_TUNE_CACHE (default
 * ~/.cache/cugmres_b200/autotune.txt); CUGMRES_AUTOTUNE=0 keeps shape 0. */
int cugmres_matvec_shapes(const cg_ctx *ctx, int precision, int *shapes);

/* y = A x.  precision CG_PREC_FP64: x, y are cg_c128 arrays; CG_PREC_MIXED:
 * cg_c64 arrays computed with the FP32 spectrum. */
int cugmres_matvec(cg_ctx *ctx, const void *x, void *y, int precision);
/* y = A^T x = x - diag(c) G x (G symmetric), the operator of PyGMRES
 * matvec(..., transpose=True) (PyGMRES/GMRES.py:47-57) and of the reference's
 * adjoint/gradient solve (CUDA_GMRES/GMRES.cuh:97-111, mask applied at the
 * crop, GMRES_kernels.cuh:305-326).  A^H x = conj(A^T conj(x)). */
int cugmres_matvec_transpose(cg_ctx *ctx, const void *x, void *y, int precision);
/* r = b - A x in FP64; *rel = ||r|| / ||b|| (either output may be NULL). */
int cugmres_residual(cg_ctx *ctx, const cg_c128 *b, const cg_c128 *x, cg_c128 *r, double *rel);

/* Solves A x = b.  x holds x0 on entry (unless opts->zero_x0) and the
 * solution on return.  res_hist (may be NULL) receives up to res_hist_len
 * relative residuals: [0] = ||b - A x0|| / ||b||, [i] = estimate after step i. */
int cugmres_solve(cg_ctx *ctx, const cg_c128 *b, cg_c128 *x, const cg_opts *opts, double *res_hist,
                  int res_hist_len, cg_result *result);

/* One independent system of a batched sweep (pointers host or device). */
typedef struct {
    int N;
    const cg_c128 *g_block; /* N x N Green's block (cugmres_green_block), or NULL:
                               the GFIEM block of k0, h built on the GPU      */
    const double *chi;      /* N x N contrast                              */
    double chi_scale;       /* A = I - G diag(chi_scale * chi)             */
    const cg_c128 *b;       /* right-hand side                             */
    cg_c128 *x;             /* x0 on entry (unless opts->zero_x0), solution */
    double k0, h;           /* wavenumber and cell size (used when g_block is NULL) */
} cg_system;

/* Solves nsys independent systems (any mix of grid sizes) on `device` with
 * `nworkers` concurrent contexts, each with its own stream; systems are taken
 * largest grid first.  The batched counterpart of the reference's sweep over
 * sizes and repetitions (CUDA_GMRES/launch_GMRES.cuh:88-235).  results[i]
 * holds system i's status, iterations, residuals and latency (operator set-up
 * plus solve, seconds).  Returns CG_OK unless a context could not be created
 * or a CUDA error occurred; per-system convergence is in results[i].status. */
int cugmres_solve_batch(int device, int nsys, const cg_system *systems, const cg_opts *opts, int nworkers,
                        cg_result *results);

/* Solves nsys independent systems in lockstep buckets -- the batched
 * counterpart of the reference's serial sweep over sizes and repetitions
 * (CUDA_GMRES/launch_GMRES.cuh:88-235), which solves one system per call.
 * Systems are grouped by grid side N (largest first), ordered by difficulty
 * (optical size N k0 h sqrt(1 + max chi)), and cut into buckets of at most
 * max_bucket systems (0: as many as fit in half of the free device memory).
 * Every kernel of an Arnoldi step is one launch for the whole bucket; each
 * restart cycle of a bucket is one CUDA-graph replay; systems that stop early
 * skip the rest of their bucket's launches.  results[i].seconds is the time
 * from the start of system i's bucket (its operator set-up included) to the
 * cycle boundary at which it finished.  Supports CG_PREC_FP64 and CG_PREC_MIXED,
 * CG_ORTHO_DCGS2, no preconditioner, A x = b; other options return
 * CG_ERR_NOT_IMPLEMENTED.
 * Per-system convergence is in results[i].status. */
int cugmres_solve_buckets(int device, int nsys, const cg_system *systems, const cg_opts *opts, int max_bucket,
                          cg_result *results);

/* Per-phase device timing of cugmres_solve, the counterpart of the reference's
 * clock_gettime step stamps (CUDA_GMRES/GMRES.cuh:39-445, labels in
 * launch_GMRES.cuh:245-307): CUDA events recorded between kernel groups on the
 * context's stream, plus the algorithmic HBM bytes each phase moves
 * (e = element bytes of the phase's precision, n = N*N):
 *   MATVEC    Arnoldi operator application, 16 n e per matvec
 *   DOTS      V^H w for k+1 basis vectors, (k+2) n e per launch
 *   AXPY      w -= V h, (k+3) n e per launch
 *   SMALL     Givens / back-substitution / cycle bookkeeping (no bulk bytes)
 *   UPDATE    x += V y, (k + 2 * 16/e) n e per cycle
 *   RESIDUAL  FP64 r = b - A x per cycle, 16 n 16 (model of one FP64 matvec)
 * Enabling resets the counters; they accumulate over solves while enabled. */
enum { CG_PHASE_MATVEC = 0, CG_PHASE_DOTS, CG_PHASE_AXPY, CG_PHASE_SMALL, CG_PHASE_UPDATE, CG_PHASE_RESIDUAL,
       CG_PHASE_PRECOND, CG_NPHASES };
typedef struct {
    double ms;          /* summed device time                 */
    double bytes;       /* summed algorithmic bytes           */
    long long launches; /* kernel groups timed                */
} cg_phase_stats;
int cugmres_profile(cg_ctx *ctx, int enable);
int cugmres_profile_read(cg_ctx *ctx, cg_phase_stats *out /* CG_NPHASES entries */);

/* Drop-in for the reference's Fast_GMRES_with_CUDA (CUDA_GMRES/GMRES.cuh:22-35):
 * same iteration semantics (exactly maxiter Arnoldi steps, no restart,
 * absolute `tolerance` gating the first step, the reference's Givens
 * formula, residual history of maxiter+1 absolute estimates), complex64 in and
 * out.  Instead of the pre-transformed spectrum, cuFFT plan and BLAS handles
 * it takes the spatial circulant G_prep ((2N-1)^2, the array the reference
 * transforms at CUDA_GMRES/launch_GMRES.cuh:138-142) and the contrast
 * `chi_value` (the reference's CHI macro, CUDA_GMRES/GMRES_kernels.cuh:19) applied where
 * mask != 0.  rhs may be NULL for the reference's plane wave exp(-i k row).
 * The arithmetic is FP64 (precision = CG_PREC_FP64) or the mixed path. */
int cugmres_fast_gmres(const cg_c64 *g_prep, const unsigned char *mask, cg_c64 *solution, float *actual_residual,
                       unsigned int *gmres_n, float tolerance, int *res_vs_tol, unsigned int maxiter, unsigned int N,
                       float chi_value, const cg_c64 *rhs, int precision);

/* Allocation-free y = A x (FP64) for callers that cannot allocate device
 * memory -- for example a plug-in inside a host application whose GPU memory
 * is owned entirely by its own pool allocator, or a latency-critical loop that
 * cannot afford the implicit device synchronisation of cudaMalloc/cudaFree.
 * No counterpart in the reference (its matvec allocates through cuFFT plans and
 * the solver cudaMallocs per call).  It builds the spectrum from g_block and
 * applies A = I - G diag(chi_scale * chi) to x, using only a fixed scratch
 * array compiled into the library (about 7.9 MB per GPU, held until exit).
 *   - N <= CUGMRES_NOALLOC_MAX_N, otherwise CG_ERR_INVALID (use cugmres_matvec);
 *   - g_block (N x N), chi (N x N), x and y must be device memory of the current
 *     device, otherwise CG_ERR_INVALID;
 *   - the first call on a device looks up the scratch array's address (once per
 *     device) and keeps it for the life of the process; make that call before
 *     any stream capture, and do not use the library across a cudaDeviceReset;
 *   - calls share the scratch array: calls whose GPU work overlaps (other
 *     streams or host threads) race, so serialise them on one stream;
 *   - the work is enqueued on `stream` (a cudaStream_t, NULL = default stream);
 *     y is ready once the stream reaches it. */
#define CUGMRES_NOALLOC_MAX_N 256
int cugmres_matvec_noalloc(int N, const cg_c128 *g_block, const double *chi, double chi_scale, const cg_c128 *x,
                           cg_c128 *y, void *stream);

/* ---------------------------------------------------------------------------
 * Learned preconditioner: a spectral-convolution network (Fourier neural
 * operator: lift 4 -> 32 channels, 4 Fourier layers of 32 channels keeping
 * 2*16 x 16 modes, projection 32 -> 128 -> 2) that maps (chi, k0 h, r) to an
 * estimate of A^{-1} r.  M(r) = r + s * net(0.1 chi, k0 h, r / s), s = rms(r).
 * BF16 activations and tensor-core weights (FP32 accumulation), FP32 master
 * parameters and Adam.  No counterpart in the reference.
 *
 * Arrays are [batch, H, W] row-major; chi FP32, r / x / z complex64, k0h FP32
 * [batch]; host or device pointers.  H >= 32, 32 <= W <= 1024.  A network is
 * used by one host thread at a time; it must not be trained while a context
 * it is attached to is solving.
 * ------------------------------------------------------------------------- */
typedef struct cg_fno cg_fno;

typedef struct {
    int layers, width, modes1, modes2, hidden, in_features;
    long long num_params; /* length of the flat FP32 parameter vector            */
    long long steps;      /* optimiser steps taken since the parameters were set */
} cg_fno_info;

int cugmres_fno_create(cg_fno **net, int device, unsigned long long seed);
void cugmres_fno_destroy(cg_fno *net);
int cugmres_fno_info(const cg_fno *net, cg_fno_info *info);
/* on = 1 (default): every Fourier layer has its pointwise path W_l; on = 0:
 * the last layer is spectral only (v_4 = b_3 + S_3(v_3), W_3 unused and its
 * gradient 0), so the correction the network adds is band-limited before the
 * projection. */
int cugmres_fno_set_local_last(cg_fno *net, int on);
/* Flat FP32 parameters, in order: P [32 x 4], p [32]; per layer l = 0..3:
 * R_l [32 k1][16 k2][32 in][32 out] complex (re, im), W_l [32 out x 32 in],
 * b_l [32]; Q1 [128 x 32], bq1 [128], Q2 [2 x 128], bq2 [2].  set_params
 * also resets the optimiser state. */
int cugmres_fno_get_params(cg_fno *net, float *params);
int cugmres_fno_set_params(cg_fno *net, const float *params);
/* z = M(r) for a batch. */
int cugmres_fno_forward(cg_fno *net, int batch, int H, int W, const float *chi, const float *k0h, const cg_c64 *r,
                        cg_c64 *z);
/* Loss L = (1/batch) sum_b ||net_b - t_b||^2 / ||t_b||^2 with t = (x - r) / s
 * (x: the solution of A x = r) and its gradient (flat, like the parameters;
 * grad may be NULL). */
int cugmres_fno_loss_grad(cg_fno *net, int batch, int H, int W, const float *chi, const float *k0h,
                          const cg_c64 *r, const cg_c64 *x, float *loss, float *grad);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the loss above. */
int cugmres_fno_train_step(cg_fno *net, int batch, int H, int W, const float *chi, const float *k0h,
                           const cg_c64 *r, const cg_c64 *x, float lr, float *loss);
/* Training with a caller-defined loss: forward_train computes z = M(r) and
 * keeps what the backward pass needs; backward takes dL/dM (complex64
 * [batch, H, W], as d/dRe + i d/dIm), writes the flat gradient (grad may be
 * NULL) and, for lr > 0, takes one Adam step.  Any other network call in
 * between discards the kept batch. */
int cugmres_fno_forward_train(cg_fno *net, int batch, int H, int W, const float *chi, const float *k0h,
                              const cg_c64 *r, cg_c64 *z);
int cugmres_fno_backward(cg_fno *net, const cg_c64 *dm, float *grad, float lr);
/* Attach (net != NULL) or detach the network to a context's solves;
 * k0h = k0 * h of the operator set with cugmres_set_operator, whose chi /
 * chi_scale give the contrast.  N of the operator must satisfy 32 <= N <= 1024. */
int cugmres_set_preconditioner(cg_ctx *ctx, cg_fno *net, double k0h);

/* C = A B^T on the tcgen05 tensor cores: A [M x K], B [N x K] BF16 row-major
 * (raw bits), C [M x N] FP32; N, K in {32, 128}; host pointers.  The
 * self-test of the kernel the network's channel mixing runs on. */
int cugmres_gemm_bf16(int device, long long M, int N, int K, const uint16_t *A, const uint16_t *B, float *C);

#ifdef __cplusplus
}
#endif

#endif /* CUGMRES_H */
