/* Host stand-in for <cuda_runtime.h>, used only to compile the reference's
 * kernels.cuh / helper_math.cuh / givens.cuh as plain host C++ for the oracle
 * pin.  Kernels become ordinary functions that the harness calls once per
 * (block, thread); floating-point atomics become plain read-modify-writes
 * (the P2G launch runs serially, in index order), the integer counter atomic
 * stays atomic. */
#pragma once
#include <math.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>
#define __host__
#define __device__
#define __global__
#define __constant__
#define __forceinline__ inline
struct ref_dim3 { unsigned x = 0, y = 0, z = 0; };
extern thread_local ref_dim3 blockIdx, threadIdx, blockDim;
inline double atomicAdd(double *a, double v) { double o = *a; *a = o + v; return o; }
inline float atomicAdd(float *a, float v) { float o = *a; *a = o + v; return o; }
inline int atomicAdd(int *a, int v) { return __atomic_fetch_add(a, v, __ATOMIC_RELAXED); }
using std::min;
using std::max;
typedef int cudaError_t;
