// Internal interface of the learned preconditioner (spectral-convolution
// network) used by the solver translation unit.  Public entry points are the
// cugmres_fno_* functions of include/cugmres.h.
#pragma once
#include <cuda_runtime.h>

struct cg_fno;

namespace cg {
namespace fno {

// Make the network ready for N x N single-vector applications with the
// given k0 h: workspace, tensor maps, twiddle tables.  May allocate and
// synchronise (call before the Arnoldi launches are enqueued).
int prepare(cg_fno *net, int N, float k0h);

// z = M(r) = r + rms(r) * net(chi, k0h, r / rms(r)) for one N x N vector,
// enqueued on `s` (after prepare(net, N, k0h)).  prec 0: r, z complex128;
// prec 1: complex64.  chi is the N x N contrast (FP32, device).  Every
// kernel returns at once while *gate != 0 (gate may be null).
int apply(cg_fno *net, cudaStream_t s, int N, int prec, const void *r, const float *chi, float k0h, void *z,
          const int *gate);

// CUDA device the network lives on.
int device_of(const cg_fno *net);

// Device error flag of the tensor-core kernels (bounded waits that ran out).
int check_error(cg_fno *net);

}  // namespace fno
}  // namespace cg
