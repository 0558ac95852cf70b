// Complex helpers and small device utilities shared by every cugmres kernel.
//
// Complex numbers are stored interleaved (re, im) as CUDA's double2 / float2,
// the layout of the reference's cuComplex (CUDA_GMRES/GMRES_kernels.cuh) and of
// numpy complex128 / complex64, so one 128-bit load moves one FP64 complex (or
// two FP32 complex values).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cg {

template <typename R> struct cplx_of;
template <> struct cplx_of<double> { typedef double2 type; };
template <> struct cplx_of<float> { typedef float2 type; };

template <typename C> struct real_of;
template <> struct real_of<double2> { typedef double type; };
template <> struct real_of<float2> { typedef float type; };

template <typename C>
__host__ __device__ __forceinline__ C mk(typename real_of<C>::type re, typename real_of<C>::type im) {
    C r;
    r.x = re;
    r.y = im;
    return r;
}
template <typename C> __host__ __device__ __forceinline__ C czero() { return mk<C>(0, 0); }
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    return mk<C>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }

// Multiply-accumulate with every real product fused into its addition: four
// FMAs per complex value (a + b * c written out as products and sums compiles
// to a multiply, an FMA and an add per component).
__device__ __forceinline__ double fma_r(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_r(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// acc + a * b
template <typename C> __device__ __forceinline__ C cfma(C acc, C a, C b) {
    return mk<C>(fma_r(-a.y, b.y, fma_r(a.x, b.x, acc.x)), fma_r(a.y, b.x, fma_r(a.x, b.y, acc.y)));
}
// acc - a * b
template <typename C> __device__ __forceinline__ C cfms(C acc, C a, C b) {
    return mk<C>(fma_r(a.y, b.y, fma_r(-a.x, b.x, acc.x)), fma_r(-a.y, b.x, fma_r(-a.x, b.y, acc.y)));
}
template <typename C>
__host__ __device__ __forceinline__ C cscale(C a, typename real_of<C>::type s) { return mk<C>(a.x * s, a.y * s); }
template <typename C> __host__ __device__ __forceinline__ typename real_of<C>::type cnorm2(C a) {
    return a.x * a.x + a.y * a.y;
}

__device__ __forceinline__ float2 to_c(float2 a, float2) { return a; }
__device__ __forceinline__ double2 to_c(double2 a, double2) { return a; }
__device__ __forceinline__ float2 to_c(double2 a, float2) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_c(float2 a, double2) { return make_double2((double)a.x, (double)a.y); }

// Warp-wide sum of a double / float with a fixed butterfly order (deterministic).
template <typename R> __device__ __forceinline__ R warp_sum(R v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Error-free transformations for the compensated FP32 sums (Ogita, Rump and
// Oishi, "Accurate sum and dot product", SIAM J. Sci. Comput. 26(6), 2005):
// TwoSum gives s + e == a + b exactly, TwoProduct (via FMA) gives p + e == a * b.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = a + b;
    float z = s - a;
    e = (a - (s - z)) + (b - z);
}
__device__ __forceinline__ void two_prod(float a, float b, float &p, float &e) {
    p = a * b;
    e = fmaf(a, b, -p);
}

// A compensated FP32 accumulator: value = hi + lo, with lo collecting every
// rounding error of the additions and products folded in (Dot2).
struct Acc2f {
    float hi, lo;
    __device__ __forceinline__ void zero() { hi = 0.f; lo = 0.f; }
    __device__ __forceinline__ void add_prod(float a, float b) {
        float p, ep, s, es;
        two_prod(a, b, p, ep);
        two_sum(hi, p, s, es);
        hi = s;
        lo += ep + es;
    }
    __device__ __forceinline__ void add(float a) {
        float s, es;
        two_sum(hi, a, s, es);
        hi = s;
        lo += es;
    }
    __device__ __forceinline__ void add_acc(const Acc2f &o) {
        float s, es;
        two_sum(hi, o.hi, s, es);
        hi = s;
        lo += es + o.lo;
    }
    __device__ __forceinline__ float value() const { return hi + lo; }
};

__device__ __forceinline__ Acc2f warp_sum(Acc2f v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Acc2f t;
        t.hi = __shfl_xor_sync(0xffffffffu, v.hi, o);
        t.lo = __shfl_xor_sync(0xffffffffu, v.lo, o);
        v.add_acc(t);
    }
    return v;
}

}  // namespace cg
