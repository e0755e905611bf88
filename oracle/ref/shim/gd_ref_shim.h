// Host stand-ins for the few CUDA device builtins that the reference's collision headers name, so
// that g++ can compile those headers unchanged.  The host entry points in ref_host.cpp never reach
// code that uses threadIdx/blockIdx/atomicAdd; min(double, double) is the only one evaluated.
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>

static inline double min(double a, double b) { return std::fmin(a, b); }
static inline double max(double a, double b) { return std::fmax(a, b); }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
static const uint3 threadIdx = {0u, 0u, 0u};
static const uint3 blockIdx = {0u, 0u, 0u};
static const dim3 blockDim = dim3(1u, 1u, 1u);
template <typename T>
static inline T atomicAdd(T *address, T value) {
    T old = *address;
    *address = old + value;
    return old;
}
static inline double __longlong_as_double(long long v) {
    double d;
    std::memcpy(&d, &v, sizeof(d));
    return d;
}
static inline long long __double_as_longlong(double d) {
    long long v;
    std::memcpy(&v, &d, sizeof(v));
    return v;
}
static inline unsigned long long atomicCAS(unsigned long long *a, unsigned long long cmp, unsigned long long v) {
    unsigned long long old = *a;
    if (old == cmp) *a = v;
    return old;
}
