// Host construction of the symmetric BTTB Green's-function block.
//
// Reference: Green_matrix_create_MKL
// (MKL_GMRES_test_09122019/source/loop_functions.h:128-168) and the NumPy
// get_green_matrix (PyGMRES/GMRES.py:20-27): g(i, j) = (i/4) H0^(1)(k r_ij)
// with r_ij = sqrt((i - 1/2)^2 + j^2), i.e. -y0/4 + i j0/4, the argument in
// float with k = 2*3.14f/(N/6.f) (parameters.h:19) and the value stored as
// complex8.  The GFIEM construction uses the physical cell size h, the h^2
// quadrature weight and the disk-averaged self term.
#include <math.h>
#include <stddef.h>

#include "../../include/cugmres.h"

extern "C" int cugmres_green_block(int kind, int N, double k0, double h, cg_c128 *out) {
    if (N < 1 || out == nullptr) return CG_ERR_INVALID;
    if (kind == CG_GREEN_REFERENCE) {
        const float k = (2 * 3.14f) / ((float)N / 6.f);
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) {
                const float t = sqrtf(powf((float)i - 0.5f, 2.f) + powf((float)j, 2.f));
                const float kr = k * t;
                cg_c128 v;
                v.re = (double)(float)(-0.25 * y0((double)kr));
                v.im = (double)(float)(0.25 * j0((double)kr));
                out[(size_t)i * N + j] = v;
            }
        return CG_OK;
    }
    if (kind == CG_GREEN_PYGMRES) {
        if (!(k0 > 0.0)) return CG_ERR_INVALID;
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) {
                const double z = k0 * sqrt((double)i * i + ((double)j - 0.5) * ((double)j - 0.5));
                cg_c128 v;
                v.re = -0.25 * y0(z);
                v.im = 0.25 * j0(z);
                out[(size_t)i * N + j] = v;
            }
        return CG_OK;
    }
    if (kind != CG_GREEN_HELMHOLTZ) return CG_ERR_INVALID;
    if (!(k0 > 0.0) || !(h > 0.0)) return CG_ERR_INVALID;
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            cg_c128 v;
            if (i == 0 && j == 0) {
                // (i pi a / (2 k0)) H1(k0 a) - 1/k0^2, the integral of (i/4) H0(k0 r) over
                // the disk of area h^2 (pi a^2 = h^2)
                const double a = h / sqrt(pi);
                const double z = k0 * a;
                const double f = pi * a / (2.0 * k0);
                v.re = -f * y1(z) - 1.0 / (k0 * k0);
                v.im = f * j1(z);
            } else {
                const double z = k0 * h * sqrt((double)i * i + (double)j * j);
                v.re = -0.25 * y0(z) * h * h;
                v.im = 0.25 * j0(z) * h * h;
            }
            out[(size_t)i * N + j] = v;
        }
    return CG_OK;
}
