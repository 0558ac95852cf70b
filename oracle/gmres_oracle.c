/* CPU oracle for the parity tests of cugmres_b200.  TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's CPU GMRES path (the MKL twin of
 * the CUDA solver, MKL_GMRES_test_09122019/source), with its own FFT in
 * place of MKL DFTI.  It is the checker, never the thing measured or shipped:
 * only tests/, the smoke check and bench.py's CPU-baseline leg load it; the
 * product library (cugmres_b200/csrc) neither links nor calls it.
 *
 * Parity is pinned against the reference's own fixtures by tests/test_oracle_*.py:
 *   - the complex64 solution of the MKL run (N=256, maxiter=44),
 *   - the G_prep_{32,64} circulants and the cylinder masks,
 *   - the Mie-series relative-error plateau (0.2381 at N=256),
 *   - the reference's NumPy matvec (PyGMRES/GMRES.py:47-57) on seeded inputs.
 *
 * Build (no MKL needed): make -C oracle   ->  oracle/_build/liboracle.so
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* complex128 instantiation: or_*_z */
#define REAL double
#define CPLX double complex
#define SFX(name) name##_z
#include "oracle_impl.h"
#undef REAL
#undef CPLX
#undef SFX

/* complex64 instantiation: or_*_c */
#define REAL float
#define CPLX float complex
#define SFX(name) name##_c
#include "oracle_impl.h"
#undef REAL
#undef CPLX
#undef SFX

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* Green's-function block of the reference, Green_matrix_create_MKL
 * (loop_functions.h:128-168): g(i, j) = -y0(kr)/4 + i j0(kr)/4 with
 * kr = k sqrt((i - 1/2)^2 + j^2), evaluated as the reference does: the
 * argument in float arithmetic with k = 2*3.14f/(N/6.f) (parameters.h:19),
 * the Bessel functions in double, the result rounded to float when
 * round_to_float is set (the reference stores complex8). */
void or_green_block_reference(int N, int round_to_float, double complex *g)
{
    const float k = (2 * 3.14f) / ((float)N / 6.f);
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            float t = sqrtf(powf((float)i - 0.5f, 2.f) + powf((float)j, 2.f));
            float kr = k * t;
            double re = -0.25 * y0((double)kr);
            double im = 0.25 * j0((double)kr);
            if (round_to_float) { re = (float)re; im = (float)im; }
            g[(size_t)i * N + j] = re + I * im;
        }
}

/* Green's-function block of the GFIEM operator A = I - k0^2 G diag(chi) on a
 * uniform grid of cell size h: off the diagonal G(d) = (i/4) H0(k0 h |d|) h^2;
 * the self term integrates (i/4) H0(k0 r) over the disk of area h^2,
 * (i pi a / (2 k0)) H1(k0 a) - 1/k0^2 with pi a^2 = h^2.  H_n = J_n + i Y_n
 * (first kind Hankel), from the C library's double j0/y0/j1/y1. */
void or_green_block_helmholtz(int N, double k0, double h, double complex *g)
{
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            double complex v;
            if (i == 0 && j == 0) {
                double a = h / sqrt(M_PI);
                double z = k0 * a;
                double f = M_PI * a / (2.0 * k0);
                v = (-f * y1(z) - 1.0 / (k0 * k0)) + I * (f * j1(z));
            } else {
                double z = k0 * h * sqrt((double)i * i + (double)j * j);
                v = (-0.25 * y0(z) + I * 0.25 * j0(z)) * h * h;
            }
            g[(size_t)i * N + j] = v;
        }
}

/* Mixed-precision GMRES with iterative refinement: the outer loop is double
 * (true residual r = b - A x with the complex128 matvec, update x += beta d),
 * each inner correction is one complex64 Arnoldi cycle of length
 * inner_restart on r / ||r||, stopped when its estimate reaches inner_tol.
 * Givens data, the triangular solve and the accumulation of d = V y are double.
 * outer_hist[o] = true relative residual before outer step o.
 * Returns 0 converged, 1 budget exhausted, 2 stagnation (an inner cycle that
 * made no progress). */
int or_gmres_ir(int N, int L, const double complex *ghat, const double *chi,
                const double complex *b, double complex *x, int inner_restart,
                double inner_tol, double tol, int max_outer, int max_inner_total,
                int rotation, double *outer_hist, int *outer_steps,
                int *inner_total, double *true_res)
{
    const size_t n = (size_t)N * N;
    const size_t LL = (size_t)L * L;
    const int m = inner_restart;
    float complex *ghat_c = (float complex *)malloc(sizeof(float complex) * LL);
    float *chi_c = (float *)malloc(sizeof(float) * n);
    for (size_t e = 0; e < LL; e++) ghat_c[e] = (float complex)ghat[e];
    for (size_t e = 0; e < n; e++) chi_c[e] = (float)chi[e];
    float complex *V = (float complex *)malloc(sizeof(float complex) * n * (size_t)(m + 1));
    double complex *r = (double complex *)malloc(sizeof(double complex) * n);
    double complex *y = (double complex *)malloc(sizeof(double complex) * (size_t)m);
    double *ihist = (double *)malloc(sizeof(double) * (size_t)m);
    const double nb = (double)nrm2_z(n, b);
    int o = 0, tot = 0, status = 1;
    double tr = 0;
    for (;;) {
        or_matvec_z(N, L, ghat, chi, x, b, r);
        double beta = (double)nrm2_z(n, r);
        tr = beta / nb;
        outer_hist[o] = tr;
        if (tr <= tol) { status = 0; break; }
        if (o >= max_outer || tot >= max_inner_total) { status = 1; break; }
        for (size_t e = 0; e < n; e++) V[e] = (float complex)(r[e] / beta);
        int brk = 0;
        int k = arnoldi_cycle_c(N, L, ghat_c, chi_c, V, 1.0, m, 1.0, inner_tol, 1,
                                rotation, max_inner_total - tot, ihist, y, &brk);
        tot += k;
        for (int j = 0; j < k; j++) {
            const float complex *vj = V + (size_t)j * n;
            double complex c = beta * y[j];
#pragma omp parallel for schedule(static)
            for (long long e = 0; e < (long long)n; e++) x[e] += c * (double complex)vj[e];
        }
        o++;
        if (k == 0) { status = 2; break; }
    }
    *outer_steps = o;
    *inner_total = tot;
    *true_res = tr;
    free(ghat_c); free(chi_c); free(V); free(r); free(y); free(ihist);
    return status;
}
