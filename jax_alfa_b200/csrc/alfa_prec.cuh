// Storage precision of one build of the engine.
//
// The engine sources (transforms, line passes, physical kernels, the step
// driver) are compiled twice: once with real = double into namespace
// alfa::f64 (the FP64 drop-in) and once with -DALFA_BUILD_FP32, real = float, into
// alfa::f32 (the FP32 and mixed-precision forms).  Fields, spectra and
// transforms use `real`; the parts that stay FP64 in every build (plane
// sums and means, the beta quintic roots, the surface-layer (MOST) planes,
// the pressure tridiagonal solve and its zero mode, profiles and forcing
// series) are written with `double` explicitly.
#pragma once
#include <cuda_runtime.h>

#ifdef ALFA_BUILD_FP32
#define ALFA_PREC f32
#else
#define ALFA_PREC f64
#endif

namespace alfa {
namespace ALFA_PREC {

#ifdef ALFA_BUILD_FP32
typedef float real;
typedef float2 cd;  // complex of real: (re, im)
__host__ __device__ __forceinline__ cd mkc(real x, real y) { return make_float2(x, y); }
#else
typedef double real;
typedef double2 cd;
__host__ __device__ __forceinline__ cd mkc(real x, real y) { return make_double2(x, y); }
#endif

// Level and row of linear index i of a field whose fastest extent is n:
// 32-bit unsigned division (engine_init keeps every padded field below 2^32
// elements; a 64-bit division costs ~10x the instructions of the kernels'
// memory traffic per element).
__host__ __device__ __forceinline__ int zof(size_t i, int n) {
  return (int)((unsigned)i % (unsigned)n);
}
__host__ __device__ __forceinline__ size_t rof(size_t i, int n) {
  return (size_t)((unsigned)i / (unsigned)n);
}

}  // namespace ALFA_PREC
}  // namespace alfa
