/* Precision-templated body of the CPU oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * Included twice by gmres_oracle.c: once with REAL=double (suffix _z) and once
 * with REAL=float (suffix _c).  Nothing here is product code; the CUDA path in
 * cugmres_b200/csrc never links or calls it.  Only tests/, the smoke check and
 * bench.py's CPU-baseline leg load the resulting liboracle.so.
 *
 * Reference being restated (paths inside the reference project, prefix
 * "Benchmarks of CUDA-based GMRES Solver .../"):
 *   MKL_GMRES_test_09122019/source/MKL_GMRES.h:3-395       FFT_GMRES_with_MKL
 *   MKL_GMRES_test_09122019/source/loop_functions.h:57-82   extend_by_zeros_MKL
 *   MKL_GMRES_test_09122019/source/loop_functions.h:128-168 Green_matrix_create_MKL
 *   MKL_GMRES_test_09122019/source/loop_functions.h:229-295 _2D_to_1D_[compared_]MKL
 *   MKL_GMRES_test_09122019/source/loop_functions.h:549-689 Givens rotation kernels
 *   MKL_GMRES_test_09122019/source/loop_functions.h:690-705 G_x_fft_matvec
 *   MKL_GMRES_test_09122019/source/loop_functions.h:761-775 mkl_Solve_LES
 * MKL itself is absent; its DFTI / BLAS / LAPACK calls are restated from their
 * documented semantics: a full 2D complex DFT (own Stockham FFT below), cdotc
 * = sum conj(x) y, scnrm2 = 2-norm, cgemm = matrix product, getrf/getrs = LU with
 * partial pivoting and the matching triangular solves.
 */

/* ---------------------------------------------------------------- FFT plan */
/* Complex product written out in real arithmetic (the same four products and
 * two sums as C99's operator, without its Annex G NaN recovery, which the
 * compiler otherwise calls out of the FFT's inner loops). */
#define SFX_CMUL(a, b) __builtin_complex((REAL)(creal(a) * creal(b) - cimag(a) * cimag(b)), \
                                         (REAL)(creal(a) * cimag(b) + cimag(a) * creal(b)))

typedef struct {
    int L;
    int nrad;
    int rad[40];
    CPLX *tw;       /* tw[m] = exp(-2 pi i m / L), m = 0..L-1, computed in double     */
    CPLX *stw[2];   /* per-stage tables, [0] forward, [1] inverse: stage s at offset  */
    int off[40];    /* off[s], entry r Ns + k = w^(k r L/(Ns R)) (k < Ns, r < R)      */
} SFX(plan_t);

static void SFX(plan_init)(SFX(plan_t) *p, int L)
{
    p->L = L;
    p->nrad = 0;
    int r = L;
    while (r % 8 == 0) { p->rad[p->nrad++] = 8; r /= 8; }
    while (r % 4 == 0) { p->rad[p->nrad++] = 4; r /= 4; }
    while (r % 2 == 0) { p->rad[p->nrad++] = 2; r /= 2; }
    while (r % 3 == 0) { p->rad[p->nrad++] = 3; r /= 3; }
    for (int f = 5; r > 1; f += 2) {
        while (r % f == 0) { p->rad[p->nrad++] = f; r /= f; }
    }
    p->tw = (CPLX *)malloc(sizeof(CPLX) * (size_t)L);
    for (int m = 0; m < L; m++) {
        double a = -2.0 * M_PI * (double)m / (double)L;
        p->tw[m] = (REAL)cos(a) + I * (REAL)sin(a);
    }
    size_t tot = 0;
    int Ns = 1;
    for (int s = 0; s < p->nrad; s++) {
        p->off[s] = (int)tot;
        tot += (size_t)p->rad[s] * Ns;
        Ns *= p->rad[s];
    }
    p->stw[0] = (CPLX *)malloc(sizeof(CPLX) * (tot ? tot : 1));
    p->stw[1] = (CPLX *)malloc(sizeof(CPLX) * (tot ? tot : 1));
    Ns = 1;
    for (int s = 0; s < p->nrad; s++) {
        const int R = p->rad[s];
        const int step = L / (Ns * R);
        for (int q = 0; q < R; q++)
            for (int k = 0; k < Ns; k++) {
                /* the same table entry the plain loop indexes: (k r step) mod L */
                const CPLX w = p->tw[(int)(((long long)k * q * step) % L)];
                p->stw[0][p->off[s] + q * Ns + k] = w;
                p->stw[1][p->off[s] + q * Ns + k] = conj(w);
            }
        Ns *= R;
    }
}

static void SFX(plan_free)(SFX(plan_t) *p)
{
    free(p->tw);
    free(p->stw[0]);
    free(p->stw[1]);
    p->tw = p->stw[0] = p->stw[1] = NULL;
}

/* 4-point DFT, sign = -1 forward, +1 inverse. */
static inline void SFX(dft4)(const CPLX *v, CPLX *V, int sign)
{
    CPLX t0 = v[0] + v[2], t1 = v[0] - v[2];
    CPLX t2 = v[1] + v[3], t3 = v[1] - v[3];
    /* multiply t3 by -i (forward) or +i (inverse) */
    CPLX t3r = (sign < 0) ? __builtin_complex((REAL)cimag(t3), (REAL)-creal(t3))
                          : __builtin_complex((REAL)-cimag(t3), (REAL)creal(t3));
    V[0] = t0 + t2;
    V[2] = t0 - t2;
    V[1] = t1 + t3r;
    V[3] = t1 - t3r;
}

/* One length-L transform of contiguous data `a` (result left in `a`), `b` is
 * scratch of length L.  Stockham auto-sort: stage with radix R and span Ns
 * reads a[j + r L/R], twiddles by w^(k r L/(Ns R)) with k = j mod Ns, does an
 * R-point DFT and writes b[(j/Ns) Ns R + k + q Ns].  sign = -1 forward,
 * +1 inverse (unnormalised). */
static void SFX(fft1d)(const SFX(plan_t) *p, CPLX *a, CPLX *b, int sign)
{
    const int L = p->L;
    CPLX *src = a, *dst = b;
    int Ns = 1;
    CPLX v[64], V[64];
    const CPLX *stw = p->stw[sign > 0 ? 1 : 0];
    for (int s = 0; s < p->nrad; s++) {
        const int R = p->rad[s];
        const int LR = L / R;
        const CPLX *ws = stw + p->off[s];
        for (int jb = 0; jb < LR; jb += Ns) {
            for (int k = 0; k < Ns; k++) {
                const int j = jb + k;
                v[0] = src[j];
                for (int r = 1; r < R; r++) v[r] = SFX_CMUL(src[j + r * LR], ws[r * Ns + k]);
                if (R == 2) {
                    V[0] = v[0] + v[1];
                    V[1] = v[0] - v[1];
                } else if (R == 4) {
                    SFX(dft4)(v, V, sign);
                } else if (R == 8) {
                    /* two 4-point DFTs of the even and odd samples, joined with
                     * the 8th roots of unity: V[q] = a[q] + w8^q b[q],
                     * V[q+4] = a[q] - w8^q b[q] */
                    CPLX e4[4] = {v[0], v[2], v[4], v[6]}, o4[4] = {v[1], v[3], v[5], v[7]};
                    CPLX a4[4], b4[4];
                    SFX(dft4)(e4, a4, sign);
                    SFX(dft4)(o4, b4, sign);
                    const REAL h = (REAL)0.70710678118654752440;
                    const REAL sg = sign < 0 ? (REAL)-1 : (REAL)1;
                    CPLX w1 = __builtin_complex(h, sg * h), w3 = __builtin_complex(-h, sg * h);
                    CPLX t1 = SFX_CMUL(b4[1], w1), t3 = SFX_CMUL(b4[3], w3);
                    CPLX t2 = __builtin_complex((REAL)(-sg * cimag(b4[2])), (REAL)(sg * creal(b4[2])));
                    V[0] = a4[0] + b4[0];
                    V[4] = a4[0] - b4[0];
                    V[1] = a4[1] + t1;
                    V[5] = a4[1] - t1;
                    V[2] = a4[2] + t2;
                    V[6] = a4[2] - t2;
                    V[3] = a4[3] + t3;
                    V[7] = a4[3] - t3;
                } else {
                    for (int q = 0; q < R; q++) {
                        CPLX acc = 0;
                        for (int r = 0; r < R; r++) {
                            int m = ((r * q) % R) * LR;
                            CPLX w = p->tw[m];
                            if (sign > 0) w = conj(w);
                            acc += SFX_CMUL(v[r], w);
                        }
                        V[q] = acc;
                    }
                }
                const int idxD = (j / Ns) * Ns * R + k;
                for (int q = 0; q < R; q++) dst[idxD + q * Ns] = V[q];
            }
        }
        CPLX *t = src; src = dst; dst = t;
        Ns *= R;
    }
    if (src != a) memcpy(a, src, sizeof(CPLX) * (size_t)L);
}

/* Columns are gathered OR_CB at a time so that every row access reads whole
 * cache lines. */
#define OR_CB 8

/* 2D DFT of an L x L row-major array in place: row transforms of rows
 * [0, rows_in) (the other rows must be zero on input, so their transforms are
 * zero and are skipped), then all column transforms, then -- for the inverse
 * pass of the matvec -- nothing else: only rows [0, rows_out) of the result are
 * guaranteed; with rows_in = rows_out = L this is the full transform. */
static void SFX(fft2d_rows)(const SFX(plan_t) *p, int L, CPLX *a, int sign, int rows)
{
#pragma omp parallel
    {
        CPLX *buf = (CPLX *)malloc(sizeof(CPLX) * (size_t)L);
#pragma omp for schedule(static)
        for (int i = 0; i < rows; i++) SFX(fft1d)(p, a + (size_t)i * L, buf, sign);
        free(buf);
    }
}

static void SFX(fft2d_cols)(const SFX(plan_t) *p, int L, CPLX *a, int sign)
{
#pragma omp parallel
    {
        CPLX *buf = (CPLX *)malloc(sizeof(CPLX) * (size_t)L * (OR_CB + 1));
        CPLX *scr = buf + (size_t)L * OR_CB;
#pragma omp for schedule(static)
        for (int c0 = 0; c0 < L; c0 += OR_CB) {
            const int nc = (L - c0) < OR_CB ? (L - c0) : OR_CB;
            for (int i = 0; i < L; i++)
                for (int q = 0; q < nc; q++) buf[(size_t)q * L + i] = a[(size_t)i * L + c0 + q];
            for (int q = 0; q < nc; q++) SFX(fft1d)(p, buf + (size_t)q * L, scr, sign);
            for (int i = 0; i < L; i++)
                for (int q = 0; q < nc; q++) a[(size_t)i * L + c0 + q] = buf[(size_t)q * L + i];
        }
        free(buf);
    }
}

/* Full 2D DFT of an L x L row-major array in place (rows, then columns). */
void SFX(or_fft2d)(int L, CPLX *a, int sign)
{
    SFX(plan_t) p;
    SFX(plan_init)(&p, L);
    SFX(fft2d_rows)(&p, L, a, sign, L);
    SFX(fft2d_cols)(&p, L, a, sign);
    SFX(plan_free)(&p);
}

/* Circulant spectrum of an even-symmetric BTTB kernel.  g_block[d1*N + d2]
 * holds G(d1, d2) for 0 <= d1, d2 < N; the embedding writes it and its
 * mirror images exactly as Green_matrix_create_MKL does
 * (loop_functions.h:150-163), generalised from L = 2N-1 to any L >= 2N-1
 * (entries with N <= |d| <= L-N stay zero). */
void SFX(or_spectrum)(int N, int L, const CPLX *g_block, CPLX *ghat)
{
    memset(ghat, 0, sizeof(CPLX) * (size_t)L * L);
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            CPLX v = g_block[(size_t)i * N + j];
            ghat[(size_t)i * L + j] = v;
            if (i > 0 && j > 0) ghat[(size_t)(L - i) * L + (L - j)] = v;
            if (i > 0) ghat[(size_t)(L - i) * L + j] = v;
            if (j > 0) ghat[(size_t)i * L + (L - j)] = v;
        }
    SFX(or_fft2d)(L, ghat, -1);
}

/* y = x - crop( IFFT2( ghat .* FFT2( pad(chi .* x) ) ) ) / L^2.
 * Restates G_x_fft_matvec + _2D_to_1D_MKL (loop_functions.h:57-82,270-295,
 * 690-705): pad the chi-scaled field into an L x L zero array, forward 2D DFT,
 * pointwise product with the spectrum, inverse 2D DFT, crop the N x N corner.
 * The reference splits the 1/L^2 normalisation between pad and crop; here it
 * is applied once at the crop.  If `plus_b` is non-NULL the function instead
 * returns r = b - (x - G chi x), the residual of _2D_to_1D_compared_MKL
 * (loop_functions.h:229-268) with the plane wave replaced by an explicit b. */
void SFX(or_matvec)(int N, int L, const CPLX *ghat, const REAL *chi,
                    const CPLX *x, const CPLX *plus_b, CPLX *y)
{
    CPLX *e = (CPLX *)malloc(sizeof(CPLX) * (size_t)L * L);
    SFX(plan_t) p;
    SFX(plan_init)(&p, L);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < L; i++) {
        CPLX *row = e + (size_t)i * L;
        int j = 0;
        if (i < N)
            for (; j < N; j++) row[j] = chi[(size_t)i * N + j] * x[(size_t)i * N + j];
        for (; j < L; j++) row[j] = 0;
    }
    /* forward 2D DFT: rows N..L-1 of the padded field are zero, so are their
     * row transforms; inverse: only rows 0..N-1 survive the crop.  Both
     * omissions leave every kept value bit for bit what the full transforms give. */
    SFX(fft2d_rows)(&p, L, e, -1, N);
    SFX(fft2d_cols)(&p, L, e, -1);
#pragma omp parallel for schedule(static)
    for (long long m = 0; m < (long long)L * L; m++) e[m] = SFX_CMUL(e[m], ghat[m]);
    SFX(fft2d_cols)(&p, L, e, +1);
    SFX(fft2d_rows)(&p, L, e, +1, N);
    SFX(plan_free)(&p);
    const REAL s = (REAL)(1.0 / ((double)L * (double)L));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            size_t o = (size_t)i * N + j;
            CPLX gx = e[(size_t)i * L + j] * s;
            if (plus_b) y[o] = plus_b[o] - x[o] + gx;
            else y[o] = x[o] - gx;
        }
    free(e);
}

/* ------------------------------------------------------- small BLAS pieces */
static CPLX SFX(dotc)(size_t n, const CPLX *x, const CPLX *y)
{
    /* sum conj(x) y; fixed-order per-thread partials so the result does not
     * depend on scheduling for a given thread count */
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    CPLX part[256];
    if (nt > 256) nt = 256;
    for (int t = 0; t < nt; t++) part[t] = 0;
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        size_t lo = n * (size_t)t / (size_t)nt, hi = n * (size_t)(t + 1) / (size_t)nt;
        CPLX acc = 0;
        for (size_t i = lo; i < hi; i++) acc += conj(x[i]) * y[i];
        part[t] = acc;
    }
    CPLX s = 0;
    for (int t = 0; t < nt; t++) s += part[t];
    return s;
}

static REAL SFX(nrm2)(size_t n, const CPLX *x)
{
    CPLX d = SFX(dotc)(n, x, x);
    return (REAL)sqrt((double)creal(d));
}

static void SFX(axpy)(size_t n, CPLX a, const CPLX *x, CPLX *y)
{
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; i++) y[i] += a * x[i];
}

/* LU with partial pivoting and solve of A y = rhs (A m x m row-major, copied).
 * Restates mkl_Solve_LES (loop_functions.h:761-775): LAPACKE_cgetrf on the
 * column-major view of the row-major HH followed by cgetrs('T'), which solves
 * HH y = cc. Returns 0 or the 1-based index of a zero pivot (getrf's info). */
static int SFX(lu_solve)(int m, const CPLX *A_in, CPLX *rhs)
{
    CPLX *A = (CPLX *)malloc(sizeof(CPLX) * (size_t)m * m);
    memcpy(A, A_in, sizeof(CPLX) * (size_t)m * m);
    int info = 0;
    for (int k = 0; k < m; k++) {
        int p = k;
        double best = cabs(A[(size_t)k * m + k]);
        for (int r = k + 1; r < m; r++) {
            double v = cabs(A[(size_t)r * m + k]);
            if (v > best) { best = v; p = r; }
        }
        if (best == 0.0) { if (!info) info = k + 1; continue; }
        if (p != k) {
            for (int c = 0; c < m; c++) {
                CPLX t = A[(size_t)k * m + c];
                A[(size_t)k * m + c] = A[(size_t)p * m + c];
                A[(size_t)p * m + c] = t;
            }
            CPLX t = rhs[k]; rhs[k] = rhs[p]; rhs[p] = t;
        }
        for (int r = k + 1; r < m; r++) {
            CPLX f = A[(size_t)r * m + k] / A[(size_t)k * m + k];
            if (f == 0) continue;
            for (int c = k; c < m; c++) A[(size_t)r * m + c] -= f * A[(size_t)k * m + c];
            rhs[r] -= f * rhs[k];
        }
    }
    for (int k = m - 1; k >= 0; k--) {
        CPLX s = rhs[k];
        for (int c = k + 1; c < m; c++) s -= A[(size_t)k * m + c] * rhs[c];
        rhs[k] = (A[(size_t)k * m + k] != 0) ? s / A[(size_t)k * m + k] : 0;
    }
    free(A);
    return info;
}

/* ------------------------------------------------ reference-faithful GMRES */
/* Restates FFT_GMRES_with_MKL (MKL_GMRES.h:3-395) step for step:
 *   r0 = b - A x0, res[0] = ||r0||, v0 = r0 * (1/||r0||)        (:70-110)
 *   if ||r0|| > tol (absolute):                                  (:119)
 *     iteration 0: w = A v0, H00 = <v0,w>, w -= H00 v0,
 *       H10 = ||w||, v1 = w + (1/H10 - 1) w, Jtotal = J0          (:121-200)
 *     for i = 1 .. maxiter-1 (no early exit):                     (:204-335)
 *       w = A v_i; modified Gram-Schmidt over j = 0..i;
 *       H(i+1,i) = ||w||; v_{i+1} = w + (1/H(i+1,i) - 1) w;
 *       Htemp = Jtotal H; rotation J from Htemp(i,i), Htemp(i+1,i)
 *       (J = [[a/rho, b/rho], [-conj(b)/rho, a/rho]], a NOT conjugated);
 *       Jtotal = J Jtotal; res[i+1] = res[0] |Jtotal(i+1, 0)|
 *     HH = (Jtotal H)[:m,:m], cc = res[0] Jtotal[:m, 0]            (:338-365)
 *     m == 1: y = cc / HH; else LU solve; x += V y                 (:366-384)
 *   *res_vs_tol = res[GMRES_i - 1] > tol                           (:387)
 * H is stored row-major with leading dimension maxiter as in the reference.
 * The matvec is or_matvec (an explicit b replaces the built-in plane wave).
 * Returns the LU info (0 on success). */
int SFX(or_gmres_reference)(int N, int L, const CPLX *ghat, const REAL *chi,
                            const CPLX *b, CPLX *x, int maxiter, REAL tol,
                            REAL *res, int *gmres_n, int *res_vs_tol)
{
    const size_t n = (size_t)N * N;
    const int m1 = maxiter + 1;
    CPLX *V = (CPLX *)malloc(sizeof(CPLX) * n * (size_t)m1);
    CPLX *H = (CPLX *)calloc((size_t)m1 * maxiter, sizeof(CPLX));
    CPLX *J = (CPLX *)calloc((size_t)m1 * m1, sizeof(CPLX));
    CPLX *col = (CPLX *)malloc(sizeof(CPLX) * (size_t)m1);
    int info = 0;
    int it = 0;

    SFX(or_matvec)(N, L, ghat, chi, x, b, V); /* r0 = b - A x0 */
    res[0] = SFX(nrm2)(n, V);
    const REAL r0 = res[0];
    const REAL inv = (REAL)1 / r0;
    for (size_t e = 0; e < n; e++) V[e] *= inv;

    if (r0 > tol) {
        for (int d = 0; d < m1; d++) J[(size_t)d * m1 + d] = 1;
        for (it = 0; it < maxiter; it++) {
            CPLX *vi = V + (size_t)it * n, *w = V + (size_t)(it + 1) * n;
            SFX(or_matvec)(N, L, ghat, chi, vi, NULL, w);
            for (int j = 0; j <= it; j++) {
                CPLX h = SFX(dotc)(n, V + (size_t)j * n, w);
                H[(size_t)j * maxiter + it] = h;
                SFX(axpy)(n, -h, V + (size_t)j * n, w);
            }
            REAL beta = SFX(nrm2)(n, w);
            H[(size_t)(it + 1) * maxiter + it] = beta;
            CPLX sc = (REAL)1 / beta - (REAL)1;
            SFX(axpy)(n, sc, w, w);
            /* Htemp column it = Jtotal(0..it+1, 0..it+1) * H(0..it+1, it) */
            for (int r = 0; r <= it + 1; r++) {
                CPLX acc = 0;
                for (int c = 0; c <= it + 1; c++) acc += J[(size_t)r * m1 + c] * H[(size_t)c * maxiter + it];
                col[r] = acc;
            }
            CPLX a = col[it], bb = col[it + 1];
            REAL rho = (REAL)sqrt((double)(creal(a) * creal(a) + creal(bb) * creal(bb) +
                                           cimag(a) * cimag(a) + cimag(bb) * cimag(bb)));
            CPLX g00 = a / rho, g01 = bb / rho, g10 = -conj(bb) / rho, g11 = a / rho;
            /* Jtotal = J Jtotal: only rows it and it+1 change */
            for (int c = 0; c <= it + 1; c++) {
                CPLX u = J[(size_t)it * m1 + c], v = J[(size_t)(it + 1) * m1 + c];
                J[(size_t)it * m1 + c] = g00 * u + g01 * v;
                J[(size_t)(it + 1) * m1 + c] = g10 * u + g11 * v;
            }
            res[it + 1] = r0 * (REAL)cabs(J[(size_t)(it + 1) * m1 + 0]);
        }
        const int m = it; /* == maxiter */
        CPLX *HH = (CPLX *)malloc(sizeof(CPLX) * (size_t)m * m);
        CPLX *cc = (CPLX *)malloc(sizeof(CPLX) * (size_t)m);
        for (int r = 0; r < m; r++) {
            for (int c = 0; c < m; c++) {
                CPLX acc = 0;
                for (int q = 0; q <= m; q++) acc += J[(size_t)r * m1 + q] * H[(size_t)q * maxiter + c];
                HH[(size_t)r * m + c] = acc;
            }
            cc[r] = J[(size_t)r * m1 + 0] * r0;
        }
        if (m == 1) {
            REAL dom = creal(HH[0]) * creal(HH[0]) + cimag(HH[0]) * cimag(HH[0]);
            cc[0] = cc[0] * conj(HH[0]) / dom;
        } else if (m > 1) {
            info = SFX(lu_solve)(m, HH, cc);
        }
        for (int j = 0; j < m; j++) SFX(axpy)(n, cc[j], V + (size_t)j * n, x);
        free(HH);
        free(cc);
    }
    *gmres_n = it;
    *res_vs_tol = (it > 0) ? (res[it - 1] > tol) : (res[0] > tol);
    free(V); free(H); free(J); free(col);
    return info;
}

/* --------------------------------------------- restarted GMRES(m), general */
/* One Arnoldi cycle of restarted GMRES, the reference method generalised with
 * what its entry point lacks (restart, early exit on a relative residual, a
 * proper complex rotation):
 *   ortho    0 = modified Gram-Schmidt (as MKL_GMRES.h:225-247)
 *            1 = classical Gram-Schmidt with one reorthogonalisation (CGS2)
 *   rotation 0 = the reference's formula J = [[a/rho, s], [-s, a/rho]]
 *                (loop_functions.h:630-689; not unitary for complex a)
 *            1 = unitary Givens J = [[conj(a)/rho, s], [-s, a/rho]]
 * Rotations are kept as (c, s) pairs and applied to each new Hessenberg
 * column, which equals the reference's Htemp = Jtotal H column (MKL_GMRES.h:
 * 275-289) without forming Jtotal.  The residual estimate |g_{k+1}| is the
 * same for both rotation formulas.  V[0] must hold r / beta on entry.  The
 * Givens data, g and the triangular solve are double whatever REAL is.
 * Writes y (k coefficients, x += V y), returns k; *brk is set on breakdown;
 * res_out[q] = |g_{q+1}| / nb for q < k. */
static int SFX(arnoldi_cycle)(int N, int L, const CPLX *ghat, const REAL *chi,
                              CPLX *V, double beta, int m, double nb, double tol,
                              int ortho, int rotation, int steps_left,
                              double *res_out, double complex *y, int *brk)
{
    const size_t n = (size_t)N * N;
    double complex *R = (double complex *)calloc((size_t)(m + 1) * m, sizeof(double complex));
    double complex *cs = (double complex *)malloc(sizeof(double complex) * (size_t)m);
    double *sn = (double *)malloc(sizeof(double) * (size_t)m);
    double complex *g = (double complex *)calloc((size_t)(m + 1), sizeof(double complex));
    double complex *h = (double complex *)malloc(sizeof(double complex) * (size_t)(m + 1));
    CPLX *hp = (CPLX *)malloc(sizeof(CPLX) * (size_t)(m + 1));
    g[0] = beta;
    *brk = 0;
    int k = 0, done = 0;
    for (k = 0; k < m && !done; k++) {
        CPLX *w = V + (size_t)(k + 1) * n;
        SFX(or_matvec)(N, L, ghat, chi, V + (size_t)k * n, NULL, w);
        for (int q = 0; q <= k + 1; q++) h[q] = 0;
        if (ortho == 0) {
            for (int j = 0; j <= k; j++) {
                CPLX hj = SFX(dotc)(n, V + (size_t)j * n, w);
                h[j] += hj;
                SFX(axpy)(n, -hj, V + (size_t)j * n, w);
            }
        } else {
            for (int pass = 0; pass < 2; pass++) {
                for (int j = 0; j <= k; j++) hp[j] = SFX(dotc)(n, V + (size_t)j * n, w);
                for (int j = 0; j <= k; j++) {
                    h[j] += hp[j];
                    SFX(axpy)(n, -hp[j], V + (size_t)j * n, w);
                }
            }
        }
        double hk1 = (double)SFX(nrm2)(n, w);
        h[k + 1] = hk1;
        if (hk1 > 0) {
            REAL invh = (REAL)(1.0 / hk1);
            for (size_t e = 0; e < n; e++) w[e] *= invh;
        } else {
            *brk = 1;
        }
        for (int j = 0; j < k; j++) {
            double complex a = h[j], bb = h[j + 1];
            double complex cj = (rotation == 1) ? conj(cs[j]) : cs[j];
            h[j] = cj * a + sn[j] * bb;
            h[j + 1] = -sn[j] * a + cs[j] * bb;
        }
        double complex a = h[k];
        double bb = creal(h[k + 1]);
        double rho = hypot(cabs(a), bb);
        double complex c;
        double s;
        if (rho == 0) { c = 1; s = 0; } else { c = a / rho; s = bb / rho; }
        cs[k] = c; sn[k] = s;
        double complex cc = (rotation == 1) ? conj(c) : c;
        h[k] = cc * a + s * bb;
        h[k + 1] = 0;
        g[k + 1] = -s * g[k];
        g[k] = cc * g[k];
        for (int q = 0; q <= k; q++) R[(size_t)q * m + k] = h[q];
        res_out[k] = cabs(g[k + 1]) / nb;
        if (res_out[k] <= tol || k + 1 >= steps_left || *brk) done = 1;
    }
    for (int q = k - 1; q >= 0; q--) {
        double complex s = g[q];
        for (int c = q + 1; c < k; c++) s -= R[(size_t)q * m + c] * y[c];
        y[q] = (R[(size_t)q * m + q] != 0) ? s / R[(size_t)q * m + q] : 0;
    }
    free(R); free(cs); free(sn); free(g); free(h); free(hp);
    return k;
}

/* Restarted GMRES(m) driver: each cycle recomputes the true residual
 * b - A x (as the reference's r0 step, MKL_GMRES.h:70-88), runs one Arnoldi
 * cycle and adds V y to x.  res_hist[0] = ||b - A x0|| / ||b||, res_hist[it]
 * = residual estimate after `it` iterations.  A cycle ends when the estimate
 * reaches tol; the next true residual confirms it, otherwise another cycle
 * starts.  Returns 0 converged, 1 not converged within maxiter, 2 breakdown
 * without convergence. */
int SFX(or_gmres)(int N, int L, const CPLX *ghat, const REAL *chi,
                  const CPLX *b, CPLX *x, int restart, int maxiter, double tol,
                  int ortho, int rotation, double *res_hist, int *iters,
                  int *cycles, double *true_res)
{
    const size_t n = (size_t)N * N;
    const int m = restart;
    CPLX *V = (CPLX *)malloc(sizeof(CPLX) * n * (size_t)(m + 1));
    CPLX *r = (CPLX *)malloc(sizeof(CPLX) * n);
    double complex *y = (double complex *)malloc(sizeof(double complex) * (size_t)m);
    const double nb = (double)SFX(nrm2)(n, b);
    int it = 0, cyc = 0, status = 1;
    double tr = 0;
    for (;;) {
        SFX(or_matvec)(N, L, ghat, chi, x, b, r);
        double beta = (double)SFX(nrm2)(n, r);
        tr = beta / nb;
        if (it == 0) res_hist[0] = tr;
        if (tr <= tol) { status = 0; break; }
        if (it >= maxiter) { status = 1; break; }
        cyc++;
        for (size_t e = 0; e < n; e++) V[e] = r[e] * (REAL)(1.0 / beta);
        int brk = 0;
        int k = SFX(arnoldi_cycle)(N, L, ghat, chi, V, beta, m, nb, tol, ortho,
                                   rotation, maxiter - it, res_hist + it + 1, y, &brk);
        it += k;
        for (int j = 0; j < k; j++) {
            const CPLX *vj = V + (size_t)j * n;
            double complex yj = y[j];
#pragma omp parallel for schedule(static)
            for (long long e = 0; e < (long long)n; e++)
                x[e] = (CPLX)((double complex)x[e] + yj * (double complex)vj[e]);
        }
        if (brk) {
            SFX(or_matvec)(N, L, ghat, chi, x, b, r);
            tr = (double)SFX(nrm2)(n, r) / nb;
            status = (tr <= tol) ? 0 : 2;
            break;
        }
    }
    *iters = it;
    *cycles = cyc;
    *true_res = tr;
    free(V); free(r); free(y);
    return status;
}
