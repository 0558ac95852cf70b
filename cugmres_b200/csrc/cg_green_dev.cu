// Device construction of the symmetric BTTB Green's-function block, so that
// the whole operator set-up (block, embedding, spectrum) runs on the GPU and
// only chi crosses the bus.  Same formulas as the host construction in
// cg_green.cpp (Green_matrix_create_MKL, MKL_GMRES_test_09122019/source/
// loop_functions.h:128-168; get_green_matrix, PyGMRES/GMRES.py:20-27; the
// GFIEM block with the h^2 weight and the disk-averaged self term), evaluated
// with CUDA's double-precision Bessel functions j0, y0, j1, y1.
#include "../../include/cugmres.h"
#include "cg_internal.h"

namespace cg {

__global__ void k_green_block(int kind, int N, double k0, double h, double2 *__restrict__ out) {
    const long long n = (long long)N * N;
    const double pi = 3.14159265358979323846;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e / N), j = (int)(e % N);
        double2 v;
        if (kind == CG_GREEN_REFERENCE) {
            // argument in float as the reference computes it, value rounded to complex8
            const float k = (2 * 3.14f) / ((float)N / 6.f);
            const float di = (float)i - 0.5f, dj = (float)j;
            const float kr = k * sqrtf(di * di + dj * dj);
            v.x = (double)(float)(-0.25 * y0((double)kr));
            v.y = (double)(float)(0.25 * j0((double)kr));
        } else if (kind == CG_GREEN_PYGMRES) {
            const double z = k0 * sqrt((double)i * i + ((double)j - 0.5) * ((double)j - 0.5));
            v.x = -0.25 * y0(z);
            v.y = 0.25 * j0(z);
        } else if (i == 0 && j == 0) {
            // (i pi a / (2 k0)) H1(k0 a) - 1/k0^2 over the disk of area h^2
            const double a = h / sqrt(pi);
            const double z = k0 * a;
            const double f = pi * a / (2.0 * k0);
            v.x = -f * y1(z) - 1.0 / (k0 * k0);
            v.y = f * j1(z);
        } else {
            const double z = k0 * h * sqrt((double)i * i + (double)j * j);
            v.x = -0.25 * y0(z) * h * h;
            v.y = 0.25 * j0(z) * h * h;
        }
        out[e] = v;
    }
}

int launch_green_block(int kind, int N, double k0, double h, double2 *out, int sms, cudaStream_t s) {
    const long long n = (long long)N * N;
    long long g = (n + 255) / 256;
    if (g > 16LL * sms) g = 16LL * sms;
    k_green_block<<<(int)(g < 1 ? 1 : g), 256, 0, s>>>(kind, N, k0, h, out);
    return (int)cudaGetLastError();
}

}  // namespace cg
