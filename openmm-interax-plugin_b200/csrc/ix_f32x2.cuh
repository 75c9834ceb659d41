// Packed single precision: two FP32 values in one 64-bit register pair, operated on by Blackwell's packed FP32
// instructions (add/sub/mul/fma .f32x2, sm_100).  One instruction issues the operation on both values, so code that
// evaluates two independent pairs in lockstep spends half the issue slots on its FP32 arithmetic.  Each element is
// rounded exactly as the scalar instruction would round it (IEEE round to nearest even).  The special-function unit
// has no packed form: those go element by element.
#pragma once

#include "ix_common.cuh"

namespace ix {

struct F2 {
    unsigned long long v;
};

__device__ __forceinline__ F2 f2(float a, float b) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ F2 f2(float a) { return f2(a, a); }
__device__ __forceinline__ float f2x(F2 p) {
    float a;
    asm("{\n\t.reg .f32 t;\n\tmov.b64 {%0, t}, %1;\n\t}" : "=f"(a) : "l"(p.v));
    return a;
}
__device__ __forceinline__ float f2y(F2 p) {
    float b;
    asm("{\n\t.reg .f32 t;\n\tmov.b64 {t, %0}, %1;\n\t}" : "=f"(b) : "l"(p.v));
    return b;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
    F2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
    F2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
    F2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
// a * b + c with one rounding per element
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
    F2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}
__device__ __forceinline__ F2 sel2(bool cx, bool cy, F2 a, F2 b) {
    return f2(cx ? f2x(a) : f2x(b), cy ? f2y(a) : f2y(b));
}

__device__ __forceinline__ F2 ex2x2(F2 y) { return f2(ex2Approx(f2x(y)), ex2Approx(f2y(y))); }
__device__ __forceinline__ F2 rcpx2(F2 y) { return f2(rcpApprox(f2x(y)), rcpApprox(f2y(y))); }
__device__ __forceinline__ F2 rsqrtx2(F2 y) { return f2(rsqrtApprox(f2x(y)), rsqrtApprox(f2y(y))); }

// expNeg element by element: the hardware 2^y of y = -x log2(e) formed as a two-float product, with the low part
// carried negated (nLo = -yLo), which the packed instructions give without a negation: x kHi + yHi is the exact
// rounding error of yHi = -x kHi, negated.
__device__ __forceinline__ F2 expNeg2(F2 x) {
    const float kLog2eHi = 1.44269502162933349609375f;
    const float kLog2eLo = 1.925963033500011079834e-8f;
    const F2 yHi = x * f2(-kLog2eHi);
    F2 nLo = fma2(x, f2(kLog2eHi), yHi);
    nLo = fma2(x, f2(kLog2eLo), nLo);
    const F2 p = ex2x2(yHi);
    return fma2(p, nLo * f2(-0.693147180559945309f), p);
}

// exp(-r q) for the float-float rate q = qHi + qLo (a reciprocal width times log2(e), formed in double on the host),
// given as nqHi = -qHi, qHi, qLo: y = -r q as a two-float product, whose low part is carried negated as in expNeg2.
__device__ __forceinline__ F2 expNegRate2(F2 r, F2 nqHi, F2 qHi, F2 qLo) {
    const F2 yHi = r * nqHi;
    F2 nLo = fma2(r, qHi, yHi);
    nLo = fma2(r, qLo, nLo);
    const F2 p = ex2x2(yHi);
    return fma2(p, nLo * f2(-0.693147180559945309f), p);
}

// sqrtRefined element by element: r and 1/r to ~0.5 ulp.
__device__ __forceinline__ F2 sqrtRefined2(F2 r2, F2& invR) {
    const F2 y = rsqrtx2(r2);
    const F2 r0 = r2 * y;
    const F2 nres = fma2(r0, r0, r2 * f2(-1.0f));         // r0^2 - r2, the residual negated
    const F2 r = fma2(nres, y * f2(-0.5f), r0);
    const F2 i0 = rcpx2(r);
    const F2 e = fma2(r * f2(-1.0f), i0, f2(1.0f));        // 1 - r i0
    invR = fma2(i0, e, i0);
    return r;
}

}  // namespace ix
