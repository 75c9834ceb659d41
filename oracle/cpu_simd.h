// Eight-lane single-precision vectors (AVX2) and the pair terms over them: the restatement of the reference CPU
// platform's SIMD pair kernel (CpuInteraxPairForceFvec.h:254-394, instantiated with fvec8 when AVX is present,
// CpuInteraxPairForceAvx.cpp:44-48), one lane per particle of a block of eight.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY (the timed CPU baseline of bench.py); never part of the product.
//
// As in the reference's vector instantiation, a branch of the scalar terms becomes a per-lane selection: both sides
// of the Slater overlap's Taylor/closed-form switch and of the Tang-Toennies series/closed-form switch are evaluated
// (each only when some lane needs it) and blended lane by lane.
#pragma once

#include <immintrin.h>

#include <cmath>
#include <cstdint>

#include "interax_oracle.hpp"

namespace ixo {
namespace simd {

struct V8 {
    __m256 v;
    V8() : v(_mm256_setzero_ps()) {}
    V8(__m256 x) : v(x) {}
    V8(float x) : v(_mm256_set1_ps(x)) {}
    static V8 load(const float* p) { return V8(_mm256_loadu_ps(p)); }
    void store(float* p) const { _mm256_storeu_ps(p, v); }
};
inline V8 operator+(V8 a, V8 b) { return _mm256_add_ps(a.v, b.v); }
inline V8 operator-(V8 a, V8 b) { return _mm256_sub_ps(a.v, b.v); }
inline V8 operator*(V8 a, V8 b) { return _mm256_mul_ps(a.v, b.v); }
inline V8 operator/(V8 a, V8 b) { return _mm256_div_ps(a.v, b.v); }
inline V8 operator-(V8 a) { return _mm256_xor_ps(a.v, _mm256_set1_ps(-0.0f)); }
inline V8& operator+=(V8& a, V8 b) { return a = a + b; }
inline V8& operator-=(V8& a, V8 b) { return a = a - b; }
inline V8& operator*=(V8& a, V8 b) { return a = a * b; }
inline V8 operator<(V8 a, V8 b) { return _mm256_cmp_ps(a.v, b.v, _CMP_LT_OQ); }
inline V8 operator>(V8 a, V8 b) { return _mm256_cmp_ps(a.v, b.v, _CMP_GT_OQ); }
inline V8 operator&(V8 a, V8 b) { return _mm256_and_ps(a.v, b.v); }
inline V8 operator|(V8 a, V8 b) { return _mm256_or_ps(a.v, b.v); }
inline V8 andNot(V8 mask, V8 a) { return _mm256_andnot_ps(mask.v, a.v); }   // a where the mask is clear
inline V8 vmin(V8 a, V8 b) { return _mm256_min_ps(a.v, b.v); }
inline V8 vmax(V8 a, V8 b) { return _mm256_max_ps(a.v, b.v); }
inline V8 vabs(V8 a) { return _mm256_andnot_ps(_mm256_set1_ps(-0.0f), a.v); }
inline V8 vsqrt(V8 a) { return _mm256_sqrt_ps(a.v); }
inline V8 vround(V8 a) { return _mm256_round_ps(a.v, _MM_FROUND_TO_NEAREST_INT | _MM_FROUND_NO_EXC); }
// a where the mask is set, b elsewhere
inline V8 select(V8 mask, V8 a, V8 b) { return _mm256_blendv_ps(b.v, a.v, mask.v); }
inline V8 zeroUnless(V8 mask, V8 a) { return _mm256_and_ps(mask.v, a.v); }
inline bool any(V8 mask) { return _mm256_movemask_ps(mask.v) != 0; }
inline bool all(V8 mask) { return _mm256_movemask_ps(mask.v) == 0xff; }
inline float sum(V8 a) {
    __m128 s = _mm_add_ps(_mm256_castps256_ps128(a.v), _mm256_extractf128_ps(a.v, 1));
    s = _mm_add_ps(s, _mm_movehl_ps(s, s));
    s = _mm_add_ss(s, _mm_shuffle_ps(s, s, 1));
    return _mm_cvtss_f32(s);
}
inline V8 laneMask(unsigned bits) {
    const __m256i bit = _mm256_setr_epi32(1, 2, 4, 8, 16, 32, 64, 128);
    const __m256i m = _mm256_and_si256(_mm256_set1_epi32((int)bits), bit);
    return _mm256_castsi256_ps(_mm256_cmpeq_epi32(m, bit));
}

// e^x: x = n ln 2 + r with |r| <= ln 2 / 2 (ln 2 split in two parts, so that n ln 2 is exact to float), e^r by its
// Taylor polynomial of degree 7 (truncation below 6e-9 relative), 2^n through the exponent bits.  Arguments below
// -87 give 0.
inline V8 vexp(V8 x) {
    const V8 lo(-87.0f), hi(88.0f);
    const V8 under = x < lo;
    x = vmin(vmax(x, lo), hi);
    const V8 n = vround(x * V8(1.44269504088896341f));
    const V8 r = (x - n * V8(0.693145751953125f)) - n * V8(1.42860682030941723e-6f);
    V8 p(1.0f / 5040.0f);
    p = p * r + V8(1.0f / 720.0f);
    p = p * r + V8(1.0f / 120.0f);
    p = p * r + V8(1.0f / 24.0f);
    p = p * r + V8(1.0f / 6.0f);
    p = p * r + V8(0.5f);
    p = p * r + V8(1.0f);
    p = p * r + V8(1.0f);
    const __m256i e = _mm256_slli_epi32(_mm256_add_epi32(_mm256_cvtps_epi32(n.v), _mm256_set1_epi32(127)), 23);
    return andNot(under, p * V8(_mm256_castsi256_ps(e)));
}

// Slater overlap S(r; a, b) and dS/dr (InteraxPairTerms.h:167-216): the order-N Taylor expansion about l where the
// scheme says so, the closed form elsewhere, per lane.
inline void slaterOverlap(V8 r, V8 a, V8 b, const SlaterTaylorScheme& scheme, V8& S, V8& dS) {
    const V8 l = scheme.aboutSmallerWidth ? vmin(a, b) : a;
    const V8 invL = V8(1.0f) / l;
    const V8 delta = (a + b) - (l + l);
    const V8 t = delta * invL;
    const V8 x = r * invL;
    const V8 absT = vabs(t);
    const V8 taylor = (vabs(delta) < V8((float)scheme.maxDelta)) |
                      ((absT < V8((float)scheme.maxT)) & (absT * x < V8((float)scheme.maxTX)));
    V8 sT, dT, sC, dC;
    if (any(taylor)) {
        const OverlapTaylorTable& table = overlapTaylorTable();
        V8 sumValue, sumDeriv;
        for (int n = scheme.order; n >= 0; n--) {
            V8 value, deriv;
            for (int k = kTaylorTerms - 1; k >= 0; k--) {
                value = value * x + V8((float)table.value[n][k]);
                deriv = deriv * x + V8((float)table.deriv[n][k]);
            }
            sumValue = sumValue * t + value;
            sumDeriv = sumDeriv * t + deriv;
        }
        const V8 pre = vexp(-x) * invL * invL * invL * V8((float)(1.0 / M_PI));
        sT = pre * sumValue;
        dT = pre * invL * sumDeriv;
    }
    if (!all(taylor)) {
        const V8 aa = a * a, bb = b * b;
        const V8 d = bb - aa;
        const V8 invD2 = V8(1.0f) / (d * d);
        const V8 expA = vexp(-r / a), expB = vexp(-r / b);
        const V8 c = V8(4.0f) * aa * bb * invD2 / d;
        const V8 f = c * (expA - expB) + r * invD2 * (a * expA + b * expB);
        const V8 dfdr = c * (expB / b - expA / a) + invD2 * (a * expA + b * expB - r * (expA + expB));
        const V8 invR = V8(1.0f) / r;
        const V8 k8pi((float)(1.0 / (8.0 * M_PI)));
        sC = f * invR * k8pi;
        dC = (r * dfdr - f) * invR * invR * k8pi;
    }
    S = select(taylor, sT, sC);
    dS = select(taylor, dT, dC);
}

// Tang-Toennies f_6, f_8, f_10 and their derivatives (InteraxPairTerms.h:223-253): the series form below (n+1)/2.
inline void tangToennies(V8 x, V8 f[3], V8 df[3]) {
    const V8 expX = vexp(-x);
    V8 term(1.0f), partial(1.0f);
    V8 terms[11], partials[11];
    terms[0] = term;
    partials[0] = partial;
    for (int k = 1; k <= 10; k++) {
        term = term * x * V8(1.0f / k);
        partial = partial + term;
        terms[k] = term;
        partials[k] = partial;
    }
    V8 tail;
    const bool needSeries = any(x < V8(5.5f));
    if (needSeries)
        for (int k = 11; k <= 40; k++) {
            term = term * x * V8(1.0f / k);
            tail = tail + term;
        }
    for (int i = 0; i < 3; i++) {
        const int n = 6 + 2 * i;
        V8 series = tail;
        for (int k = n + 1; k <= 10; k++) series = series + terms[k];
        f[i] = select(x < V8(0.5f * (n + 1)), expX * series, V8(1.0f) - expX * partials[n]);
        df[i] = expX * terms[n];
    }
}

// Dispersion (InteraxPairTerms.h:267-293); p = m1, m2, m3, alpha, width of each side.
inline void dispersionPair(V8 r, const V8* p, const V8* q, float dampingScale, V8& energy, V8& dEdR) {
    const V8 denom = p[3] * q[0] + q[3] * p[0];
    const V8 pref = p[3] * q[3] / select(denom > V8(1e-30f), denom, V8(1e-30f));
    V8 c[3];
    c[0] = pref * p[0] * q[0];
    c[1] = V8(1.5f) * pref * (p[0] * q[1] + p[1] * q[0]);
    c[2] = pref * (V8(2.0f) * (p[0] * q[2] + p[2] * q[0]) + V8(4.2f) * p[1] * q[1]);
    const V8 dxdr = V8(2.0f * dampingScale) / (p[4] + q[4]);
    V8 f[3], df[3];
    tangToennies(dxdr * r, f, df);
    const V8 invR = V8(1.0f) / r;
    const V8 invR2 = invR * invR;
    V8 invRn = invR2 * invR2 * invR2;
    energy = V8(0.0f);
    dEdR = V8(0.0f);
    for (int i = 0; i < 3; i++) {
        energy = energy - f[i] * c[i] * invRn;
        dEdR = dEdR - c[i] * invRn * (df[i] * dxdr - V8((float)(6 + 2 * i)) * f[i] * invR);
        invRn = invRn * invR2;
    }
}

// Exchange A_i A_j S (InteraxPairTerms.h:305-312); p = amplitude, width.
inline void exchangePair(V8 r, const V8* p, const V8* q, const SlaterTaylorScheme& scheme, V8& energy, V8& dEdR) {
    V8 s, ds;
    slaterOverlap(r, p[1], q[1], scheme, s, ds);
    const V8 amp = p[0] * q[0];
    energy = amp * s;
    dEdR = amp * ds;
}

// Short range (K_i+K_j)/2 St + (L_i+L_j)/2 St^2 (InteraxPairTerms.h:325-337); p = k, l, width.
inline void shortRangePair(V8 r, const V8* p, const V8* q, const SlaterTaylorScheme& scheme, V8& energy, V8& dEdR) {
    V8 s, ds;
    slaterOverlap(r, p[2], q[2], scheme, s, ds);
    const V8 ws = p[2] + q[2];
    const V8 norm = V8((float)(8.0 * M_PI)) * ws * ws * ws;
    const V8 st = norm * s;
    const V8 k = V8(0.5f) * (p[0] + q[0]);
    const V8 l = V8(0.5f) * (p[1] + q[1]);
    energy = (k + l * st) * st;
    dEdR = (k + V8(2.0f) * l * st) * norm * ds;
}

}  // namespace simd
}  // namespace ixo
