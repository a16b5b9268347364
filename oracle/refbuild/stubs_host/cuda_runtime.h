/* Host stand-in for <cuda_runtime.h>, used only to compile the reference's
 * kernels.cuh / helper_math.cuh / givens.cuh as plain host C++ for the oracle
 * pin.  Kernels become ordinary functions that the harness calls once per
 * (block, thread); floating-point atomics are plain read-modify-writes for
 * the serial P2G launch (index order) and real atomics for the parallel one;
 * the integer counter atomic stays atomic. */
#pragma once
#include <math.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#define __host__
#define __device__
#define __global__
#define __constant__
#define __forceinline__ inline
struct ref_dim3 { unsigned x = 0, y = 0, z = 0; };
extern thread_local ref_dim3 blockIdx, threadIdx, blockDim;
/* ref_atomics_on (set by the harness): the floating-point atomics are real
 * (relaxed) atomic read-modify-writes, so that P2G may run its blocks in
 * parallel as it does on the GPU; off, they are plain adds for the serial,
 * point-ordered P2G of the golden fixtures. */
extern bool ref_atomics_on;
inline double atomicAdd(double *a, double v)
{
    if (ref_atomics_on) return std::atomic_ref<double>(*a).fetch_add(v, std::memory_order_relaxed);
    double o = *a; *a = o + v; return o;
}
inline float atomicAdd(float *a, float v)
{
    if (ref_atomics_on) return std::atomic_ref<float>(*a).fetch_add(v, std::memory_order_relaxed);
    float o = *a; *a = o + v; return o;
}
inline int atomicAdd(int *a, int v) { return __atomic_fetch_add(a, v, __ATOMIC_RELAXED); }
using std::min;
using std::max;
typedef int cudaError_t;
