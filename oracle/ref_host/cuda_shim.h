// Test infrastructure only: lets the reference's own CUDA source
// (src/octmps_kernel.cuh, included by path, never copied) compile as plain
// host C++ so that it can serve as the CPU baseline and as a check on the
// restatement in oracle/oracle.cpp.  Nothing in the product links this.
//
// Each CUDA construct the reference uses is mapped to host C++:
//  * qualifiers (__device__, __global__, __constant__) vanish; a kernel is a
//    function the driver calls once per emulated thread;
//  * blockIdx/threadIdx are thread-local, set by the driver before each call;
//  * atomics map to the GCC __atomic builtins;
//  * __ddiv_rd (round-down division, src/octmps_kernel.h:38) is computed
//    exactly from the round-to-nearest quotient and its FMA remainder;
//  * __uint2float_rz (src/octmps_kernel.cuh:17) truncates to 24 significant
//    bits before the exact conversion;
//  * rsqrt(x) is 1/sqrt(x); log, sincos, acos, sqrt are glibc's;
//  * the runtime calls the .cuh makes (cudaMemcpyToSymbol, cudaMemcpy,
//    cudaFree) become memcpy/free on host memory.
#ifndef OCTMPS_REF_CUDA_SHIM_H
#define OCTMPS_REF_CUDA_SHIM_H

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#define __device__
#define __global__
#define __host__
#define __constant__
#define __align__(n) __attribute__((aligned(n)))
#define __syncthreads() ((void)0)
#define checkCudaErrors(x) (x)
#define CUT_THREADPROC void *
#define CUT_THREADROUTINE void *(*)(void *)

struct shim_dim3 {
    unsigned int x, y, z;
};
extern thread_local shim_dim3 blockIdx;
extern thread_local shim_dim3 threadIdx;
extern shim_dim3 blockDim;
extern shim_dim3 gridDim;

typedef int cudaError_t;
enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3
};
static const cudaError_t cudaSuccess = 0;

template <typename S>
static inline cudaError_t cudaMemcpyToSymbol(S &symbol, const void *src, size_t n) {
    memcpy((void *)&symbol, src, n);
    return cudaSuccess;
}
static inline cudaError_t cudaMemcpy(void *dst, const void *src, size_t n, cudaMemcpyKind) {
    memmove(dst, src, n);
    return cudaSuccess;
}
static inline cudaError_t cudaFree(void *p) {
    free(p);
    return cudaSuccess;
}

static inline unsigned long long atomicCAS(unsigned long long *addr, unsigned long long expected,
                                           unsigned long long desired) {
    __atomic_compare_exchange_n(addr, &expected, desired, false, __ATOMIC_SEQ_CST,
                                __ATOMIC_SEQ_CST);
    return expected;  // the value seen at addr, as CUDA's atomicCAS returns
}
static inline unsigned long long atomicAdd(unsigned long long *addr, unsigned long long v) {
    return __atomic_fetch_add(addr, v, __ATOMIC_SEQ_CST);
}
static inline unsigned int atomicAdd(unsigned int *addr, unsigned int v) {
    return __atomic_fetch_add(addr, v, __ATOMIC_SEQ_CST);
}
static inline unsigned int atomicSub(unsigned int *addr, unsigned int v) {
    return __atomic_fetch_sub(addr, v, __ATOMIC_SEQ_CST);
}

static inline long long __double_as_longlong(double d) {
    long long r;
    memcpy(&r, &d, sizeof r);
    return r;
}
static inline double __longlong_as_double(long long v) {
    double r;
    memcpy(&r, &v, sizeof r);
    return r;
}

// Round-toward-minus-infinity quotient.  q = RN(a/b); r = a - q*b is exact
// (one FMA) whenever q is the correctly rounded quotient, so the sign of r
// against the sign of b says whether RN rounded up past the true quotient.
static inline double __ddiv_rd(double a, double b) {
    double q = a / b;
    if (!std::isfinite(q) || q == 0.0) return q;
    double r = std::fma(-q, b, a);
    if (r != 0.0 && ((r < 0.0) == (b > 0.0))) q = std::nextafter(q, -INFINITY);
    return q;
}

// float(u) rounded toward zero: keep the top 24 significant bits.
static inline float __uint2float_rz(unsigned int u) {
    if (u >= (1u << 24)) {
        int lead = 31 - __builtin_clz(u);
        u &= ~((1u << (lead - 23)) - 1u);
    }
    return (float)u;
}

static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }

#endif
