// Complex helpers shared by the LU kernels (double or float components).
#pragma once

#include <cuda_runtime.h>

namespace fhb {

template <class T>
struct __align__(2 * sizeof(T)) Cx {
    T re, im;
};

template <class T>
__device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class T>
__device__ __forceinline__ Cx<T> csub(Cx<T> a, Cx<T> b) {
    return {a.re - b.re, a.im - b.im};
}
// Complex division as the reference's num-complex does it.
template <class T>
__device__ __forceinline__ Cx<T> cdiv(Cx<T> a, Cx<T> b) {
    T ns = b.re * b.re + b.im * b.im;
    T re = a.re * b.re + a.im * b.im;
    T im = a.im * b.re - a.re * b.im;
    return {re / ns, im / ns};
}
// y -= f * x
template <class T>
__device__ __forceinline__ void csubmul(Cx<T> &y, Cx<T> f, Cx<T> x) {
    y.re -= f.re * x.re - f.im * x.im;
    y.im -= f.re * x.im + f.im * x.re;
}
// Load bypassing L1 (data written by other CTAs during the same kernel).
template <class T>
__device__ __forceinline__ Cx<T> ldcg(const Cx<T> *p);
template <>
__device__ __forceinline__ Cx<double> ldcg(const Cx<double> *p) {
    double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return {v.x, v.y};
}
template <>
__device__ __forceinline__ Cx<float> ldcg(const Cx<float> *p) {
    float2 v = __ldcg(reinterpret_cast<const float2 *>(p));
    return {v.x, v.y};
}

}  // namespace fhb
