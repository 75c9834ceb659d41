// Pair energies of the InteraxFF dispersion, exchange and short-range terms in single precision.
//
// Same functions as the reference (openmmapi/include/internal/InteraxPairTerms.h:167-337; CUDA snippets
// platforms/common/src/kernels/interaxDispersion.cc, interaxSlaterOverlap.cc, interaxExchange.cc,
// interaxShortRange.cc), evaluated in a form chosen for float arithmetic:
//
//  * The Slater overlap S(r; a, b) uses no Taylor/closed-form switch for the Exact method.  With a <= b,
//    h = b - a, s = a + b and delta = r h / (a b) >= 0 the closed form can be rewritten without cancellation as
//        8 pi S = e^(-r/a) [ 1/s^3 + r/(a s^3) + r^2/(2 a^2 b s^2) + phi3(delta) r^2 (r h/(a^3 b^2 s^2) - 4/(a b s^3)) ]
//    with phi_k(z) = sum_n z^n/(n+k)! (phi3 = (e^z - 1 - z - z^2/2)/z^3), which is positive and smooth in delta.
//    For equal widths it reduces to the limit e^(-x)(1 + x + x^2/3)/(64 pi a^3).  Evaluated in float it is exact to
//    a few ulp for all widths and distances, where the reference's float switch loses up to ~1e-2 near t = 0.2.
//  * The InteraxOrder2 method reproduces the export's order-2 expansion about the width of the particle with the
//    lower original index where the widths differ by less than 0.01 bohr (InteraxPairTerms.h:151-159), and is the
//    exact overlap elsewhere, which is what the reference's closed form computes there.
//  * Tang-Toennies damping keeps the reference's series/closed-form switch at x = (n+1)/2
//    (InteraxPairTerms.h:223-253), with the series truncated at k = 28, which is exact to float rounding for
//    x < 5.5.
#pragma once

#include "ix_common.cuh"
#include "ix_f32x2.cuh"
#include "overlap_taylor_table.h"

namespace ix {

constexpr float kInv8Pi = 0.0397887357729738339422f;   // 1/(8 pi)
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kOrder2MaxDelta = 0.01f * 0.0529177210903f;   // 0.01 bohr in nm

// A Slater width as float-float: the width w + wLo and its reciprocal iw + iwLo, each the double-precision value
// split into a float and the float remainder.  The low parts keep the widths' rounding out of the exponentials.
struct Width {
    float w, wLo, iw, iwLo;
};

// 8 pi S and d(8 pi S)/dr for widths A <= B (the cancellation-free form above).
__device__ __forceinline__ void overlapExact(float r, const Width& A, const Width& B, float& s8pi, float& ds8pi) {
    const float a = A.w, ia = A.iw, ib = B.iw;
    const float h = (B.w - A.w) + (B.wLo - A.wLo);
    const float s = (A.w + B.w) + (A.wLo + B.wLo);
    float is = rcpApprox(s);
    is = fmaf(is, fmaf(-s, is, 1.0f), is);
    const float is2 = is * is;
    const float is3 = is2 * is;
    const float ea = expNegScaled(r, A.iw, A.iwLo);
    (void)a;
    const float hab = h * ia * ib;          // d delta / dr
    const float d = r * hab;                 // delta >= 0
    float eP3, eP4;                          // e^(-r/a) phi3(delta), e^(-r/a) phi4(delta)
    if (d < 2.0f) {
        // phi4(d) = sum_{n=0}^{11} d^n/(n+4)!; the omitted terms are below 1e-8 relative for d < 2
        float p4 = 1.0f / 1307674368000.0f;                 // 1/15!
        p4 = fmaf(p4, d, 1.0f / 87178291200.0f);            // 1/14!
        p4 = fmaf(p4, d, 1.0f / 6227020800.0f);             // 1/13!
        p4 = fmaf(p4, d, 1.0f / 479001600.0f);              // 1/12!
        p4 = fmaf(p4, d, 1.0f / 39916800.0f);               // 1/11!
        p4 = fmaf(p4, d, 1.0f / 3628800.0f);                // 1/10!
        p4 = fmaf(p4, d, 1.0f / 362880.0f);                 // 1/9!
        p4 = fmaf(p4, d, 1.0f / 40320.0f);                  // 1/8!
        p4 = fmaf(p4, d, 1.0f / 5040.0f);                   // 1/7!
        p4 = fmaf(p4, d, 1.0f / 720.0f);                    // 1/6!
        p4 = fmaf(p4, d, 1.0f / 120.0f);                    // 1/5!
        p4 = fmaf(p4, d, 1.0f / 24.0f);                     // 1/4!
        const float p3 = fmaf(d, p4, 1.0f / 6.0f);
        eP3 = ea * p3;
        eP4 = ea * p4;
    }
    else {
        // no cancellation worth the series here: e_b - e_a (1 + d + d^2/2) loses at most a factor 3 at d = 2
        const float eb = expNegScaled(r, B.iw, B.iwLo);
        float id = rcpApprox(d);
        id = fmaf(id, fmaf(-d, id, 1.0f), id);
        eP3 = (eb - ea * fmaf(d, fmaf(0.5f, d, 1.0f), 1.0f)) * id * id * id;
        eP4 = fmaf(ea, -1.0f / 6.0f, eP3) * id;
    }
    const float c2 = ia * is3;
    const float c3 = 0.5f * ia * ia * ib * is2;
    const float k1 = h * ia * ia * ia * ib * ib * is2;
    const float k2 = 4.0f * ia * ib * is3;
    const float rk1 = r * k1;
    const float br = r * r * (rk1 - k2);
    const float dbr = r * fmaf(3.0f, rk1, -2.0f * k2);
    const float poly = fmaf(r, fmaf(r, c3, c2), is3);
    const float dpoly = fmaf(2.0f * r, c3, c2);
    const float eg = fmaf(eP3, br, ea * poly);
    const float egp = fmaf(eP3, dbr, fmaf(fmaf(-3.0f, eP4, eP3) * hab, br, ea * dpoly));
    s8pi = eg;
    ds8pi = fmaf(-eg, ia, egp);
}

// Order-2 Taylor expansion of InteraxFF about width l (l = the width of the lower-index particle), returns
// 8 pi S and its derivative.
__device__ __forceinline__ void overlapOrder2Taylor(float r, const Width& L, const Width& O, float& s8pi,
                                                    float& ds8pi) {
    const float il = L.iw;
    const float t = ((O.w - L.w) + (O.wLo - L.wLo)) * il;
    const float x = r * il;
    float sv = 0.0f, sd = 0.0f;
#pragma unroll
    for (int n = 2; n >= 0; n--) {
        float v = 0.0f, dv = 0.0f;
#pragma unroll
        for (int k = n + 2; k >= 0; k--) {
            v = fmaf(v, x, kOverlapTaylorValue[n][k]);
            dv = fmaf(dv, x, kOverlapTaylorDeriv[n][k]);
        }
        sv = fmaf(sv, t, v);
        sd = fmaf(sd, t, dv);
    }
    const float pre = expNegScaled(r, L.iw, L.iwLo) * il * il * il * (8.0f);   // 8 pi S = 8 e^-x / l^3 sum ...
    s8pi = pre * sv;
    ds8pi = pre * il * sd;
}

// 8 pi S(r) and its derivative for the widths of particles i and j, with the overlap method of the force.
// firstIsI: particle i has the lower original index (InteraxOrder2 expands about its width).
__device__ __forceinline__ void overlap8pi(float r, const Width& Wi, const Width& Wj, int method, bool firstIsI,
                                           float& s8pi, float& ds8pi) {
    if (method == 2 && fabsf((Wi.w - Wj.w) + (Wi.wLo - Wj.wLo)) < kOrder2MaxDelta) {
        if (firstIsI) overlapOrder2Taylor(r, Wi, Wj, s8pi, ds8pi);
        else overlapOrder2Taylor(r, Wj, Wi, s8pi, ds8pi);
        return;
    }
    if (Wi.w < Wj.w || (Wi.w == Wj.w && Wi.wLo <= Wj.wLo)) overlapExact(r, Wi, Wj, s8pi, ds8pi);
    else overlapExact(r, Wj, Wi, s8pi, ds8pi);
}

// ---------------------------------------------------------------------------------------------------------------------
// Pair coefficients of two parameter classes.  When a system's particles fall into few distinct parameter tuples
// (atom types), every coefficient that depends only on the two particles' parameters is computed once on the host in
// double precision and rounded to float once: C6, C8, C10 and the damping rate of the dispersion, the overlap's
// polynomial coefficients (with a <= b: 1/a, 1/b as float-float, 1/a - 1/b, 1/s^3, 1/(a s^3), 1/(2 a^2 b s^2),
// h/(a^3 b^2 s^2), 4/(a b s^3)), A_i A_j/(8 pi), (s_i + s_j)^3, (K_i + K_j)/2 and (L_i + L_j)/2.  The kernel then
// evaluates only the r-dependent part.
// ---------------------------------------------------------------------------------------------------------------------
struct PairCoef {
    float4 disp;    // C6, C8, C10, dx/dr = 2 beta/(w_i + w_j)
    float4 ovA;     // exchange overlap: 1/a, its float remainder, 1/b, its float remainder
    float4 ovB;     // 1/a - 1/b, 1/s^3, 1/(a s^3), 1/(2 a^2 b s^2)
    float4 ovC;     // h/(a^3 b^2 s^2), 4/(a b s^3), A_i A_j/(8 pi), unused
    float4 srA;     // short-range overlap, as ovA (equal to it when the two forces share widths)
    float4 srB;     // as ovB
    float4 srC;     // as ovC .x .y; (s_i + s_j)^3 of the short-range widths; unused
    float4 srK;     // (K_i + K_j)/2, (L_i + L_j)/2, unused, unused
    // the exponential rates of the packed path: q = log2(e)/width as float-float (qHi + qLo)
    float4 ovQ;     // exchange overlap: -qa float part, qa float part, qa remainder, -qb float part
    float4 ovR;     // qb float part, qb remainder, unused, unused
    float4 srQ;     // short-range overlap, as ovQ
    float4 srR;     // as ovR
};

// 8 pi S and its derivative from the coefficients (the cancellation-free form of overlapExact).
__device__ __forceinline__ void overlapFromCoef(float r, const float4& A, const float4& B, float k1, float k2,
                                                float& s8pi, float& ds8pi) {
    const float ia = A.x, hab = B.x, is3 = B.y, c2 = B.z, c3 = B.w;
    const float ea = expNegScaled(r, A.x, A.y);
    const float d = r * hab;
    float eP3, eP4;
    if (d < 2.0f) {
        float p4 = 1.0f / 1307674368000.0f;
        p4 = fmaf(p4, d, 1.0f / 87178291200.0f);
        p4 = fmaf(p4, d, 1.0f / 6227020800.0f);
        p4 = fmaf(p4, d, 1.0f / 479001600.0f);
        p4 = fmaf(p4, d, 1.0f / 39916800.0f);
        p4 = fmaf(p4, d, 1.0f / 3628800.0f);
        p4 = fmaf(p4, d, 1.0f / 362880.0f);
        p4 = fmaf(p4, d, 1.0f / 40320.0f);
        p4 = fmaf(p4, d, 1.0f / 5040.0f);
        p4 = fmaf(p4, d, 1.0f / 720.0f);
        p4 = fmaf(p4, d, 1.0f / 120.0f);
        p4 = fmaf(p4, d, 1.0f / 24.0f);
        eP3 = ea * fmaf(d, p4, 1.0f / 6.0f);
        eP4 = ea * p4;
    }
    else {
        const float eb = expNegScaled(r, A.z, A.w);
        float id = rcpApprox(d);
        id = fmaf(id, fmaf(-d, id, 1.0f), id);
        eP3 = (eb - ea * fmaf(d, fmaf(0.5f, d, 1.0f), 1.0f)) * id * id * id;
        eP4 = fmaf(ea, -1.0f / 6.0f, eP3) * id;
    }
    const float rk1 = r * k1;
    const float br = r * r * (rk1 - k2);
    const float dbr = r * fmaf(3.0f, rk1, -2.0f * k2);
    const float poly = fmaf(r, fmaf(r, c3, c2), is3);
    const float dpoly = fmaf(2.0f * r, c3, c2);
    const float eg = fmaf(eP3, br, ea * poly);
    const float egp = fmaf(eP3, dbr, fmaf(fmaf(-3.0f, eP4, eP3) * hab, br, ea * dpoly));
    s8pi = eg;
    ds8pi = fmaf(-eg, ia, egp);
}

// Damped C6/C8/C10 dispersion from the coefficients (InteraxPairTerms.h:223-293): the partial sums of the
// exponential series by Horner's rule, the series form of f_n below x = (n+1)/2.
__device__ __forceinline__ void dispersionFromCoef(float r, float invR, const float4& K, float& energy, float& dEdR) {
    const float dxdr = K.w;
    const float x = dxdr * r;
    const float expX = expNeg(x);
    const float x2 = x * x;
    const float x3 = x2 * x;
    const float t6 = x3 * x3 * (1.0f / 720.0f);
    const float t7 = t6 * x * (1.0f / 7.0f);
    const float t8 = t7 * x * (1.0f / 8.0f);
    const float t9 = t8 * x * (1.0f / 9.0f);
    const float t10 = t9 * x * (1.0f / 10.0f);
    float s6 = fmaf(x, 1.0f / 720.0f, 1.0f / 120.0f);
    s6 = fmaf(s6, x, 1.0f / 24.0f);
    s6 = fmaf(s6, x, 1.0f / 6.0f);
    s6 = fmaf(s6, x, 0.5f);
    s6 = fmaf(s6, x, 1.0f);
    s6 = fmaf(s6, x, 1.0f);
    const float s8 = (s6 + t7) + t8;
    const float s10 = (s8 + t9) + t10;
    float f6 = fmaf(-expX, s6, 1.0f), f8 = fmaf(-expX, s8, 1.0f), f10 = fmaf(-expX, s10, 1.0f);
    if (x < 5.5f) {
        float term = t10, tail = 0.0f;
#pragma unroll 1
        for (int k = 11; k <= 28; k++) {
            term = term * x * __fdividef(1.0f, (float)k);
            tail += term;
        }
        const float tail8 = (tail + t10) + t9;
        f10 = expX * tail;
        if (x < 4.5f) f8 = expX * tail8;
        if (x < 3.5f) f6 = expX * ((tail8 + t8) + t7);
    }
    const float invR2 = invR * invR;
    const float e6 = K.x * invR2 * invR2 * invR2;
    const float e8 = K.y * invR2 * invR2 * invR2 * invR2;
    const float e10 = K.z * invR2 * invR2 * invR2 * invR2 * invR2;
    energy = -fmaf(f6, e6, fmaf(f8, e8, f10 * e10));
    const float g = expX * dxdr;
    dEdR = -(e6 * fmaf(g, t6, -6.0f * f6 * invR) + e8 * fmaf(g, t8, -8.0f * f8 * invR) +
             e10 * fmaf(g, t10, -10.0f * f10 * invR));
}

// dispersionFromCoef for two pairs at once: the closed forms of both as one straight sequence (two independent
// chains for the scheduler to interleave), then the series form of f_n for a pair below x = (n+1)/2 (rare at
// interacting distances).
__device__ __forceinline__ void dispersionFromCoef2(const float r[2], const float invR[2], const float4 K[2],
                                                    float energy[2], float dEdR[2]) {
    float x[2], expX[2], t6[2], t7[2], t8[2], t9[2], t10[2], f6[2], f8[2], f10[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        x[k] = K[k].w * r[k];
        expX[k] = expNeg(x[k]);
        const float x2 = x[k] * x[k];
        const float x3 = x2 * x[k];
        t6[k] = x3 * x3 * (1.0f / 720.0f);
        t7[k] = t6[k] * x[k] * (1.0f / 7.0f);
        t8[k] = t7[k] * x[k] * (1.0f / 8.0f);
        t9[k] = t8[k] * x[k] * (1.0f / 9.0f);
        t10[k] = t9[k] * x[k] * (1.0f / 10.0f);
        float s6 = fmaf(x[k], 1.0f / 720.0f, 1.0f / 120.0f);
        s6 = fmaf(s6, x[k], 1.0f / 24.0f);
        s6 = fmaf(s6, x[k], 1.0f / 6.0f);
        s6 = fmaf(s6, x[k], 0.5f);
        s6 = fmaf(s6, x[k], 1.0f);
        s6 = fmaf(s6, x[k], 1.0f);
        const float s8 = (s6 + t7[k]) + t8[k];
        const float s10 = (s8 + t9[k]) + t10[k];
        f6[k] = fmaf(-expX[k], s6, 1.0f);
        f8[k] = fmaf(-expX[k], s8, 1.0f);
        f10[k] = fmaf(-expX[k], s10, 1.0f);
    }
#pragma unroll
    for (int k = 0; k < 2; k++)
        if (x[k] < 5.5f) {
            float term = t10[k], tail = 0.0f;
#pragma unroll 1
            for (int m = 11; m <= 28; m++) {
                term = term * x[k] * __fdividef(1.0f, (float)m);
                tail += term;
            }
            const float tail8 = (tail + t10[k]) + t9[k];
            f10[k] = expX[k] * tail;
            if (x[k] < 4.5f) f8[k] = expX[k] * tail8;
            if (x[k] < 3.5f) f6[k] = expX[k] * ((tail8 + t8[k]) + t7[k]);
        }
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float invR2 = invR[k] * invR[k];
        const float e6 = K[k].x * invR2 * invR2 * invR2;
        const float e8 = K[k].y * invR2 * invR2 * invR2 * invR2;
        const float e10 = K[k].z * invR2 * invR2 * invR2 * invR2 * invR2;
        energy[k] = -fmaf(f6[k], e6, fmaf(f8[k], e8, f10[k] * e10));
        const float g = expX[k] * K[k].w;
        dEdR[k] = -(e6 * fmaf(g, t6[k], -6.0f * f6[k] * invR[k]) + e8 * fmaf(g, t8[k], -8.0f * f8[k] * invR[k]) +
                    e10 * fmaf(g, t10[k], -10.0f * f10[k] * invR[k]));
    }
}

// overlapFromCoef for two pairs at once.  Where the warp holds both sides of the series/closed-form switch, both are
// evaluated and each pair takes its own, so that the two chains stay one straight sequence.
__device__ __forceinline__ void overlapFromCoef2(const float r[2], const float4 A[2], const float4 B[2],
                                                 const float k1[2], const float k2[2], float s8pi[2],
                                                 float ds8pi[2]) {
    float ea[2], d[2], eP3[2], eP4[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        ea[k] = expNegScaled(r[k], A[k].x, A[k].y);
        d[k] = r[k] * B[k].x;
    }
    const unsigned active = __activemask();
    const bool anySeries = __any_sync(active, d[0] < 2.0f || d[1] < 2.0f);
    const bool anyClosed = __any_sync(active, d[0] >= 2.0f || d[1] >= 2.0f);
#pragma unroll
    for (int k = 0; k < 2; k++) {
        float sP3 = 0.0f, sP4 = 0.0f, cP3 = 0.0f, cP4 = 0.0f;
        if (anySeries) {
            const float dd = fminf(d[k], 2.0f);
            float p4 = 1.0f / 1307674368000.0f;
            p4 = fmaf(p4, dd, 1.0f / 87178291200.0f);
            p4 = fmaf(p4, dd, 1.0f / 6227020800.0f);
            p4 = fmaf(p4, dd, 1.0f / 479001600.0f);
            p4 = fmaf(p4, dd, 1.0f / 39916800.0f);
            p4 = fmaf(p4, dd, 1.0f / 3628800.0f);
            p4 = fmaf(p4, dd, 1.0f / 362880.0f);
            p4 = fmaf(p4, dd, 1.0f / 40320.0f);
            p4 = fmaf(p4, dd, 1.0f / 5040.0f);
            p4 = fmaf(p4, dd, 1.0f / 720.0f);
            p4 = fmaf(p4, dd, 1.0f / 120.0f);
            p4 = fmaf(p4, dd, 1.0f / 24.0f);
            sP3 = ea[k] * fmaf(dd, p4, 1.0f / 6.0f);
            sP4 = ea[k] * p4;
        }
        if (anyClosed) {
            const float dd = fmaxf(d[k], 2.0f);
            const float eb = expNegScaled(r[k], A[k].z, A[k].w);
            float id = rcpApprox(dd);
            id = fmaf(id, fmaf(-dd, id, 1.0f), id);
            cP3 = (eb - ea[k] * fmaf(dd, fmaf(0.5f, dd, 1.0f), 1.0f)) * id * id * id;
            cP4 = fmaf(ea[k], -1.0f / 6.0f, cP3) * id;
        }
        const bool series = d[k] < 2.0f;
        eP3[k] = series ? sP3 : cP3;
        eP4[k] = series ? sP4 : cP4;
    }
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float ia = A[k].x, hab = B[k].x, is3 = B[k].y, c2 = B[k].z, c3 = B[k].w;
        const float rk1 = r[k] * k1[k];
        const float br = r[k] * r[k] * (rk1 - k2[k]);
        const float dbr = r[k] * fmaf(3.0f, rk1, -2.0f * k2[k]);
        const float poly = fmaf(r[k], fmaf(r[k], c3, c2), is3);
        const float dpoly = fmaf(2.0f * r[k], c3, c2);
        const float eg = fmaf(eP3[k], br, ea[k] * poly);
        const float egp = fmaf(eP3[k], dbr, fmaf(fmaf(-3.0f, eP4[k], eP3[k]) * hab, br, ea[k] * dpoly));
        s8pi[k] = eg;
        ds8pi[k] = fmaf(-eg, ia, egp);
    }
}

// Tang-Toennies damped C6/C8/C10 dispersion (InteraxPairTerms.h:267-293).  p = (m1, m2, m3, alpha), w the widths.
__device__ __forceinline__ void dispersionEnergy(float r, float invR, float4 pi, float4 pj, float wi, float wj,
                                                 float twoBeta, float& energy, float& dEdR) {
    const float denom = fmaxf(fmaf(pi.w, pj.x, pj.w * pi.x), 1e-30f);
    const float pref = pi.w * pj.w * __fdividef(1.0f, denom);
    const float c6 = pref * pi.x * pj.x;
    const float c8 = 1.5f * pref * fmaf(pi.x, pj.y, pi.y * pj.x);
    const float c10 = pref * fmaf(2.0f, fmaf(pi.x, pj.z, pi.z * pj.x), 4.2f * pi.y * pj.y);
    const float dxdr = twoBeta * __fdividef(1.0f, wi + wj);
    const float x = dxdr * r;
    const float expX = expNeg(x);
    float t[11];
    t[0] = 1.0f;
#pragma unroll
    for (int k = 1; k <= 10; k++) t[k] = t[k - 1] * x * (1.0f / k);
    const float s6 = (((((1.0f + t[1]) + t[2]) + t[3]) + t[4]) + t[5]) + t[6];
    const float s8 = (s6 + t[7]) + t[8];
    const float s10 = (s8 + t[9]) + t[10];
    float f6 = fmaf(-expX, s6, 1.0f), f8 = fmaf(-expX, s8, 1.0f), f10 = fmaf(-expX, s10, 1.0f);
    if (x < 5.5f) {
        // f_n = exp(-x) sum_{k>n} x^k/k! where the closed form cancels
        float term = t[10], tail = 0.0f;
#pragma unroll 1
        for (int k = 11; k <= 28; k++) {
            term = term * x * __fdividef(1.0f, (float)k);
            tail += term;
        }
        const float tail10 = tail;
        const float tail8 = (tail10 + t[10]) + t[9];
        const float tail6 = (tail8 + t[8]) + t[7];
        f10 = expX * tail10;
        if (x < 4.5f) f8 = expX * tail8;
        if (x < 3.5f) f6 = expX * tail6;
    }
    const float invR2 = invR * invR;
    const float invR6 = invR2 * invR2 * invR2;
    const float e6 = c6 * invR6, e8 = c8 * invR6 * invR2, e10 = c10 * invR6 * invR2 * invR2;
    energy = -fmaf(f6, e6, fmaf(f8, e8, f10 * e10));
    const float g = expX * dxdr;
    dEdR = -(e6 * fmaf(g, t[6], -6.0f * f6 * invR) + e8 * fmaf(g, t[8], -8.0f * f8 * invR) +
             e10 * fmaf(g, t[10], -10.0f * f10 * invR));
}

// ---------------------------------------------------------------------------------------------------------------------
// Two pairs at once in packed FP32 (F2, ix_f32x2.cuh): the class-table forms above evaluated in lockstep on two pairs
// of one lane.  Each returns what its scalar form returns, with the sign of some outputs folded away (noted per
// function) so that no packed negation is needed.  Their rounding differs from the scalar forms only where a
// product's rounding order differs; both agree with the FP64 oracle to the same bound.
// ---------------------------------------------------------------------------------------------------------------------

// dispersionFromCoef for two pairs: returns -energy (nE) and -dE/dr (nD).
__device__ __forceinline__ void dispersionFromCoefP(F2 r, F2 invR, F2 c6, F2 c8, F2 c10, F2 dxdr, F2& nE, F2& nD) {
    const F2 x = dxdr * r;
    const F2 expX = expNeg2(x);
    const F2 x2 = x * x;
    const F2 x3 = x2 * x;
    const F2 t6 = (x3 * x3) * f2(1.0f / 720.0f);
    const F2 t7 = (t6 * x) * f2(1.0f / 7.0f);
    const F2 t8 = (t7 * x) * f2(1.0f / 8.0f);
    const F2 t9 = (t8 * x) * f2(1.0f / 9.0f);
    const F2 t10 = (t9 * x) * f2(1.0f / 10.0f);
    F2 s6 = fma2(x, f2(1.0f / 720.0f), f2(1.0f / 120.0f));
    s6 = fma2(s6, x, f2(1.0f / 24.0f));
    s6 = fma2(s6, x, f2(1.0f / 6.0f));
    s6 = fma2(s6, x, f2(0.5f));
    s6 = fma2(s6, x, f2(1.0f));
    s6 = fma2(s6, x, f2(1.0f));
    const F2 s8 = (s6 + t7) + t8;
    const F2 s10 = (s8 + t9) + t10;
    const F2 nExp = expX * f2(-1.0f);
    F2 f6 = fma2(nExp, s6, f2(1.0f)), f8 = fma2(nExp, s8, f2(1.0f)), f10 = fma2(nExp, s10, f2(1.0f));
    const float xa = f2x(x), xb = f2y(x);
    if (xa < 5.5f || xb < 5.5f) {
        // the series form where the closed form cancels (rare at interacting distances)
        F2 term = t10, tail = f2(0.0f);
#pragma unroll 1
        for (int k = 11; k <= 28; k++) {
            term = (term * x) * f2(__fdividef(1.0f, (float)k));
            tail = tail + term;
        }
        const F2 tail8 = (tail + t10) + t9;
        const F2 f10s = expX * tail, f8s = expX * tail8, f6s = expX * ((tail8 + t8) + t7);
        f10 = sel2(xa < 5.5f, xb < 5.5f, f10s, f10);
        f8 = sel2(xa < 4.5f, xb < 4.5f, f8s, f8);
        f6 = sel2(xa < 3.5f, xb < 3.5f, f6s, f6);
    }
    const F2 invR2 = invR * invR;
    const F2 e6 = ((c6 * invR2) * invR2) * invR2;
    const F2 e8 = (((c8 * invR2) * invR2) * invR2) * invR2;
    const F2 e10 = ((((c10 * invR2) * invR2) * invR2) * invR2) * invR2;
    nE = fma2(f6, e6, fma2(f8, e8, f10 * e10));
    const F2 g = expX * dxdr;
    const F2 a6 = fma2(g, t6, (f6 * f2(-6.0f)) * invR);
    const F2 a8 = fma2(g, t8, (f8 * f2(-8.0f)) * invR);
    const F2 a10 = fma2(g, t10, (f10 * f2(-10.0f)) * invR);
    nD = fma2(e10, a10, fma2(e8, a8, e6 * a6));
}

// overlapFromCoef for two pairs: 8 pi S and its derivative.  A, B, k1, k2 as overlapFromCoef (packed per element);
// nqa, qa, qaLo and nqb, qb, qbLo the exponential rates (PairCoef ovQ/ovR).  `active`: the lanes of the warp that
// call it together (they agree on which forms of the series/closed-form switch to evaluate).
__device__ __forceinline__ void overlapFromCoefP(F2 r, F2 ia, F2 hab, F2 is3, F2 c2, F2 c3, F2 k1, F2 k2, F2 nqa,
                                                 F2 qa, F2 qaLo, F2 nqb, F2 qb, F2 qbLo, unsigned active, F2& s8pi,
                                                 F2& ds8pi) {
    const F2 ea = expNegRate2(r, nqa, qa, qaLo);
    const F2 d = r * hab;
    const float da = f2x(d), db = f2y(d);
    const bool seriesA = da < 2.0f, seriesB = db < 2.0f;
    const bool anySeries = __any_sync(active, seriesA || seriesB);
    const bool anyClosed = __any_sync(active, !seriesA || !seriesB);
    F2 sP3 = f2(0.0f), sP4 = f2(0.0f), cP3 = f2(0.0f), cP4 = f2(0.0f);
    if (anySeries) {
        const F2 dd = f2(fminf(da, 2.0f), fminf(db, 2.0f));
        F2 p4 = fma2(f2(1.0f / 1307674368000.0f), dd, f2(1.0f / 87178291200.0f));
        p4 = fma2(p4, dd, f2(1.0f / 6227020800.0f));
        p4 = fma2(p4, dd, f2(1.0f / 479001600.0f));
        p4 = fma2(p4, dd, f2(1.0f / 39916800.0f));
        p4 = fma2(p4, dd, f2(1.0f / 3628800.0f));
        p4 = fma2(p4, dd, f2(1.0f / 362880.0f));
        p4 = fma2(p4, dd, f2(1.0f / 40320.0f));
        p4 = fma2(p4, dd, f2(1.0f / 5040.0f));
        p4 = fma2(p4, dd, f2(1.0f / 720.0f));
        p4 = fma2(p4, dd, f2(1.0f / 120.0f));
        p4 = fma2(p4, dd, f2(1.0f / 24.0f));
        sP3 = ea * fma2(dd, p4, f2(1.0f / 6.0f));
        sP4 = ea * p4;
    }
    if (anyClosed) {
        const F2 dd = f2(fmaxf(da, 2.0f), fmaxf(db, 2.0f));
        const F2 eb = expNegRate2(r, nqb, qb, qbLo);
        F2 id = rcpx2(dd);
        id = fma2(id, fma2(dd * f2(-1.0f), id, f2(1.0f)), id);
        cP3 = (eb - ea * fma2(dd, fma2(f2(0.5f), dd, f2(1.0f)), f2(1.0f))) * ((id * id) * id);
        cP4 = fma2(ea, f2(-1.0f / 6.0f), cP3) * id;
    }
    const F2 eP3 = sel2(seriesA, seriesB, sP3, cP3), eP4 = sel2(seriesA, seriesB, sP4, cP4);
    const F2 rk1 = r * k1;
    const F2 br = (r * r) * (rk1 - k2);
    const F2 dbr = r * fma2(f2(3.0f), rk1, k2 * f2(-2.0f));
    const F2 poly = fma2(r, fma2(r, c3, c2), is3);
    const F2 dpoly = fma2(r * f2(2.0f), c3, c2);
    const F2 eg = fma2(eP3, br, ea * poly);
    const F2 egp = fma2(eP3, dbr, fma2(fma2(f2(-3.0f), eP4, eP3) * hab, br, ea * dpoly));
    s8pi = eg;
    ds8pi = fma2(eg * f2(-1.0f), ia, egp);
}

}  // namespace ix
