// Host/device portability layer for the physics headers.
//
// Every physics routine in this directory is written once and compiled twice:
// by nvcc for sm_100a (the product kernels) and by g++ for the host-side unit
// tests that check individual routines against the reference on the CPU.  The
// product library has no host execution path; the host build exists only so that
// tests can call single routines without a GPU.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define RSB_HD __host__ __device__ __forceinline__
#define RSB_D __device__ __forceinline__
#define RSB_CONST __constant__
#else
#define RSB_HD inline
#define RSB_D inline
#define RSB_CONST
#endif

#include <math.h>
#include <string.h>

namespace rsb {

// Bullet constants (LinearMath/btScalar.h) used by the algorithms restated here.
constexpr float kEpsilon = 1.1920928955078125e-07f;  // FLT_EPSILON
constexpr float kLargeFloat = 1e18f;
constexpr float kPi = 3.1415926535897932384626433832795029f;
constexpr float kTwoPi = 6.283185307179586232f;
constexpr float kHalfPi = 1.5707963267948966192f;
constexpr float kSqrt12 = 0.7071067811865475244008443621048490f;
constexpr float kInf = __builtin_huge_valf();

// Unit conversion (RocketSim BaseInc: 1 Bullet unit = 50 Unreal units).
constexpr float kUuToBt = 1.f / 50.f;
constexpr float kBtToUu = 50.f;

RSB_HD float fsqrt(float x) { return sqrtf(x); }
RSB_HD float fabsf_(float x) { return fabsf(x); }
RSB_HD float fmin_(float a, float b) { return a < b ? a : b; }
RSB_HD float fmax_(float a, float b) { return a > b ? a : b; }
RSB_HD float fclamp(float v, float lo, float hi) { return fmin_(fmax_(v, lo), hi); }
RSB_HD int imin_(int a, int b) { return a < b ? a : b; }
RSB_HD int imax_(int a, int b) { return a > b ? a : b; }

}  // namespace rsb
