// Device helpers shared by the pair and three-body kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

#include "ix_tuning.h"

namespace ix {

constexpr int kWarp = 32;
constexpr double kFixedScale = 4294967296.0;   // 2^32: the fixed-point scale of OpenMM's force buffers
constexpr float kFixedScaleF = 4294967296.0f;

// Fast reciprocal and reciprocal square root (MUFU, ~1 ulp).
__device__ __forceinline__ float rcpApprox(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrtApprox(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2Approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2Approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// exp(-x) for x >= 0 with a relative error of a few ulp over the whole range.  The argument of the hardware 2^y is
// formed as a two-float product y = -x log2(e) (Dekker splitting via FMA), so that its rounding error, which the
// exponential amplifies by |y|, is carried in the correction term instead of being lost.
__device__ __forceinline__ float expNeg(float x) {
    const float kLog2eHi = 1.44269502162933349609375f;          // log2(e) rounded to float
    const float kLog2eLo = 1.925963033500011079834e-8f;         // log2(e) - kLog2eHi
    float yHi = -x * kLog2eHi;
    float yLo = fmaf(-x, kLog2eHi, -yHi);                       // exact rounding error of the product
    yLo = fmaf(-x, kLog2eLo, yLo);
    float p = ex2Approx(yHi);
    return fmaf(p, yLo * 0.693147180559945309f, p);            // 2^yLo ~ 1 + yLo ln 2
}

// exp(-(xHi + xLo)) for a float-float argument (|xLo| << xHi).
__device__ __forceinline__ float expNegDF(float xHi, float xLo) {
    const float kLog2eHi = 1.44269502162933349609375f;
    const float kLog2eLo = 1.925963033500011079834e-8f;
    float yHi = -xHi * kLog2eHi;
    float yLo = fmaf(-xHi, kLog2eHi, -yHi);
    yLo = fmaf(-xHi, kLog2eLo, yLo);
    yLo = fmaf(-xLo, kLog2eHi, yLo);
    float p = ex2Approx(yHi);
    return fmaf(p, yLo * 0.693147180559945309f, p);
}

// exp(-r (invHi + invLo)), the exponent formed with a compensated product: the rounding of the reciprocal width
// to float, which the exponential would amplify by r/width (10 to 40 for interacting pairs) into a systematic error,
// is carried in invLo.
__device__ __forceinline__ float expNegScaled(float r, float invHi, float invLo) {
    const float xHi = r * invHi;
    const float xLo = fmaf(r, invHi, -xHi) + r * invLo;
    return expNegDF(xHi, xLo);
}

// sqrt(r2) to ~0.5 ulp: approximate reciprocal square root followed by one Newton correction of the root.
__device__ __forceinline__ float sqrtRefined(float r2, float& invR) {
    float y = rsqrtApprox(r2);
    float r = r2 * y;
    float residual = fmaf(-r, r, r2);
    r = fmaf(residual, 0.5f * y, r);
    invR = rcpApprox(r);
    invR = fmaf(invR, fmaf(-r, invR, 1.0f), invR);              // one Newton step on 1/r
    return r;
}

__device__ __forceinline__ long long toFixed(float v) { return __float2ll_rn(v * kFixedScaleF); }
__device__ __forceinline__ long long toFixedD(double v) { return __double2ll_rn(v * kFixedScale); }

__device__ __forceinline__ void atomicAddFixed(long long* p, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

// Periodic box in OpenMM's reduced form, with the reciprocal diagonal.
struct Box {
    double a[3], b[3], c[3];
    double inv[3];
    int triclinic;
};

// Minimum image of a displacement: c, then b, then a, as OpenMM's ReferenceForce::getDeltaRPeriodic does (for a
// rectangular box this is the per-component rounding).  floor(v + 0.5) as in the reference.
__device__ __forceinline__ void minimumImage(double& dx, double& dy, double& dz, const Box& box) {
    double s = floor(dz * box.inv[2] + 0.5);
    dx -= s * box.c[0];
    dy -= s * box.c[1];
    dz -= s * box.c[2];
    s = floor(dy * box.inv[1] + 0.5);
    dx -= s * box.b[0];
    dy -= s * box.b[1];
    s = floor(dx * box.inv[0] + 0.5);
    dx -= s * box.a[0];
}

// The same in single precision (used only to select candidate pairs; the interaction itself uses the double version).
struct BoxF {
    float a[3], b[3], c[3];
    float inv[3];
};
__device__ __forceinline__ void minimumImageF(float& dx, float& dy, float& dz, const BoxF& box) {
    float s = floorf(dz * box.inv[2] + 0.5f);
    dx -= s * box.c[0];
    dy -= s * box.c[1];
    dz -= s * box.c[2];
    s = floorf(dy * box.inv[1] + 0.5f);
    dx -= s * box.b[0];
    dy -= s * box.b[1];
    s = floorf(dx * box.inv[0] + 0.5f);
    dx -= s * box.a[0];
}

__device__ __forceinline__ unsigned laneMaskLt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ double warpSumD(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warpMaxF(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warpMinF(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// A named NVTX range over a host scope (the API calls, graph captures and list growth), visible in Nsight Systems
// timelines; with no profiler attached NVTX does nothing.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace ix
