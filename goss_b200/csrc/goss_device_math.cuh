// Scalar math used by the generated model code and the solver kernels.
//
// Every function has a float and a double overload.  The double overloads
// call CUDA's correctly behaved double-precision functions (the FP64 path is
// checked state for state against the FP64 CPU oracle).  The float overloads
// map to the SFU approximations (ex2/lg2/rcp/rsqrt based intrinsics) that make
// the FP32 path fast; its accuracy is checked against FP64 in the tests.
#ifndef GOSS_DEVICE_MATH_CUH
#define GOSS_DEVICE_MATH_CUH

#include <cuda_runtime.h>
#include <math.h>

namespace goss_b200 { namespace models {

__device__ __forceinline__ double gexp(double x) { return exp(x); }
__device__ __forceinline__ float gexp(float x) { return __expf(x); }
// 2^x: the hardware exponential (ex2.approx, flush-to-zero, as __expf uses) in
// FP32; exp2 in FP64.  The generator prints exp(c*x) as gexp2((c*log2 e)*x).
__device__ __forceinline__ double gexp2(double x) { return exp2(x); }
__device__ __forceinline__ float gexp2(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ double glog(double x) { return log(x); }
__device__ __forceinline__ float glog(float x) { return __logf(x); }
__device__ __forceinline__ double gsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float gsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double gfabs(double x) { return fabs(x); }
__device__ __forceinline__ float gfabs(float x) { return fabsf(x); }
__device__ __forceinline__ double gfloor(double x) { return floor(x); }
__device__ __forceinline__ float gfloor(float x) { return floorf(x); }
__device__ __forceinline__ double gceil(double x) { return ceil(x); }
__device__ __forceinline__ float gceil(float x) { return ceilf(x); }
__device__ __forceinline__ double gpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float gpow(float x, float y) { return __powf(x, y); }
__device__ __forceinline__ double gfmax(double x, double y) { return fmax(x, y); }
__device__ __forceinline__ float gfmax(float x, float y) { return fmaxf(x, y); }
__device__ __forceinline__ double gfmin(double x, double y) { return fmin(x, y); }
__device__ __forceinline__ float gfmin(float x, float y) { return fminf(x, y); }
__device__ __forceinline__ double gsin(double x) { return sin(x); }
__device__ __forceinline__ float gsin(float x) { return __sinf(x); }
__device__ __forceinline__ double gcos(double x) { return cos(x); }
__device__ __forceinline__ float gcos(float x) { return __cosf(x); }
__device__ __forceinline__ double gtan(double x) { return tan(x); }
__device__ __forceinline__ float gtan(float x) { return __tanf(x); }
__device__ __forceinline__ double gtanh(double x) { return tanh(x); }
__device__ __forceinline__ float gtanh(float x) { return tanhf(x); }

}}  // namespace goss_b200::models

namespace goss_b200 {

// phi1(x) = (e^x - 1)/x with phi1(0) = 1, in single precision.
//
// The generalised Rush-Larsen update y + b/a (e^{a h} - 1) equals
// y + b h phi1(a h).  Evaluating e^{a h} - 1 in single precision cancels
// catastrophically when |a h| is small (gating variables with time constants
// of hundreds of ms at h = 0.01 ms give |a h| ~ 1e-5, leaving ~2 correct
// digits), so the FP32 kernels use phi1 instead: for |x| < 1/4 the Taylor
// series sum_k x^k/(k+1)! truncated after x^6 (relative truncation error
// < (1/4)^7/8! < 2e-9), otherwise (e^x - 1)/x with the SFU exponential.
__device__ __forceinline__ float phi1f(float x)
{
    const float ax = fabsf(x);
    if (ax < 0.25f) {
        // Horner form of 1 + x/2 + x^2/6 + x^3/24 + x^4/120 + x^5/720 + x^6/5040
        float p = 1.0f / 5040.0f;
        p = fmaf(p, x, 1.0f / 720.0f);
        p = fmaf(p, x, 1.0f / 120.0f);
        p = fmaf(p, x, 1.0f / 24.0f);
        p = fmaf(p, x, 1.0f / 6.0f);
        p = fmaf(p, x, 0.5f);
        p = fmaf(p, x, 1.0f);
        return p;
    }
    return __fdividef(__expf(x) - 1.0f, x);
}

}  // namespace goss_b200

#endif
