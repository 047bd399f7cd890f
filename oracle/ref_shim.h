/* TEST INFRASTRUCTURE ONLY -- part of the oracle, never linked into the product.
 *
 * Host-compilation shim for the reference's CUDA kernels.  The recipe in
 * oracle/Makefile extracts the device code of the reference's .cu files (every
 * line before the host launcher, minus the CUDA runtime includes) into
 * oracle/_ref/ and compiles it with g++ with this header force-included, so
 * that each __global__ function becomes a plain C++ function evaluated for one
 * (blockIdx, threadIdx) at a time.  Arithmetic is IEEE single (or double for
 * the FP64 variant, which adds `#define float double` after this header),
 * compiled with -ffp-contract=off so that no multiply-add is fused.
 */
#ifndef SYSMAT_ORACLE_REF_SHIM_H
#define SYSMAT_ORACLE_REF_SHIM_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>
#include <chrono>
#include <math.h>

#define __device__
#define __global__
#define __host__
#define __forceinline__ inline

struct ref_uint3 { unsigned int x, y, z; };
extern thread_local ref_uint3 blockIdx;
extern thread_local ref_uint3 threadIdx;
extern thread_local ref_uint3 blockDim;

/* Crystal sub-cell counts: the recipe rewrites the reference's
 * `const unsigned int divideX = 8, divideY = 16, divideZ = 8;`
 * (PESysMatGen.cu:435) to read these, so one build covers every sub-cell grid. */
extern thread_local unsigned int ref_div[3];

/* One host thread evaluates one (row, col[, slice]) cell at a time, so the
 * device atomics become plain read-modify-writes in loop order.  As with
 * CUDA's atomicAdd(float*, float), the value is first converted to the
 * target's type (the scatter kernels pass a double expression,
 * scatter.cu:1427, :1924). */
template <class T, class U> inline T atomicAdd(T* p, U v) { T old = *p; *p = old + (T)v; return old; }
inline unsigned int atomicOr(unsigned int* p, unsigned int v) { unsigned int old = *p; *p = old | v; return old; }

typedef int cudaError_t;
#define cudaSuccess 0
inline const char* cudaGetErrorString(int) { return "host shim"; }

#endif
