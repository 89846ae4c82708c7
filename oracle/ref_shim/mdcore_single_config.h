/* Configuration of the single-precision mdcore build (FPTYPE=float), as the
 * reference's cmake generates it: scalar paths, no MPI, no CUDA. */
#pragma once
#include <float.h>
#include <math.h>
#define MX_OPENMP 0
#define MX_OPENMP_BONDS 0
#define MX_OPENMP_INTEGRATOR 0
#define MX_VECTORIZE_FLUX 0
#define MX_VECTORIZE_FORCE 0
#define MX_VECTORIZE_BONDS 0
#define MX_VECTORIZE_INTEGRATOR 0
#define MX_THREADING 1
#define MX_AVX2 0
#define MX_AVX 0
#define MX_SSE42 0
#define MX_SIMD_SIZE 4
#ifndef FPTYPE_DEFINED
typedef float FPTYPE;
#define FPTYPE_EPSILON FLT_EPSILON
#define FPTYPE_ONE 1.0f
#define FPTYPE_ZERO 0.0f
#define FPTYPE_TWO 2.0f
#define FPTYPE_SQRT sqrtf
#define FPTYPE_FMAX fmaxf
#define FPTYPE_FMIN fminf
#define FPTYPE_FABS fabsf
#define FPTYPE_SINGLE
#define FPTYPE_DEFINED
#endif
