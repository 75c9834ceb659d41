// Fused pair kernel: the dispersion, exchange and short-range terms of every interacting pair in one pass over the
// tile list (the reference runs them as snippets of OpenMM's nonbonded kernel in one pass,
// platforms/common/src/CommonInteraxKernels.cpp:139-219, kernels interaxPairBegin.cc / interaxPairEnd.cc).
//
// Warps take tiles from a counter in global memory until none is left (dynamic balance).  Per tile:
//   1. staging: the 32 i particles and the tile's 32 j particles are written to shared memory as
//      float-float offsets from the i-block's center (the double-precision difference split into a float and its
//      float remainder).  In large rectangular boxes each j particle is placed at its minimum image relative to the
//      block center here, once, instead of per pair;
//   2. queue: the tile's row masks (built with the list, with the list's skin) give the candidate pairs.  The
//      displacement of a pair is formed as (xj - xi) + (lo_j - lo_i) (the precision of the double difference, without
//      double arithmetic) and tested against the exact cutoff (borderline cases decided in double).  Where the pairs
//      are costly (per-particle parameters, soft core, switch or order-2 overlap), each lane first keeps the
//      candidates of its row within the cutoff, so that the expensive phase runs with every lane on a pair that
//      interacts; on the lean class-table path the compute phase tests each candidate instead.  The pairs of each row
//      are written to a per-warp queue at the row's offset (a warp prefix sum of the row counts); the column masks
//      are the transpose of the row masks;
//   3. compute phase, in rounds of kPairRound queued pairs: each lane takes one pair, forms its displacement (the
//      same operations), evaluates the three terms in float and stores the pair force in shared memory;
//   4. gather: lane i sums the forces of its row (contiguous in the queue), lane j those of its column (located from
//      the column mask and the row offsets), in a fixed order and without atomics; both go to the global 64-bit
//      fixed-point force buffer (scale 2^32) after the tile.  Each tile's energies, summed per lane and then over
//      the lanes in double, are written to a per-tile slot and summed in a fixed order afterwards.  Results do not
//      depend on which warp ran which tile.
#pragma once

#include "ix_nblist.cuh"
#include "ix_pair_math.cuh"

namespace ix {

// Periodic box as float-float vectors (for minimum images of float-float displacements).
struct BoxFF {
    float a[3], b[3], c[3];
    float aLo[3], bLo[3], cLo[3];
    float inv[3];
    int triclinic;
};

struct PairTermConfig {
    int termMask;                // bit t: term t is evaluated in this call
    float lambda[3];
    float softShift[3];          // (1 - lambda) R^6 of each term, 0 = no soft core
    int useSwitch[3];
    float switchDist[3], invSwitchWidth[3];
    float twoBeta;               // 2 x damping scale of the dispersion
    int overlapMethod[3];
    int shareOverlap;            // exchange and short-range widths are identical for every particle
    int useCutoff, periodic;
    float cutoff2;
    double cutoff;
    Box box;
    BoxFF boxff;
    int alchOnlyBit;             // nonzero: only the pairs with exactly one particle carrying this alchemical flag bit
    int coefShared;              // the class-pair table is read from its copy in shared memory
};

struct PairBuffers {
    const float4* p0;            // sorted: m1, m2, m3, alpha
    const float4* p1;            // sorted: dispersion width, amplitude A, K, L
    const float4* p2;            // sorted: exchange width, 1/width, short-range width, 1/width
    const float4* p3;            // sorted: the float remainders of p2's four values (float-float widths)
    const int* flags;            // sorted
    long long* forceFixed;       // 3 x np, sorted order, SoA
    double* taskEnergy;          // 3 per task, summed in a fixed order afterwards
    unsigned long long* pairCount;
    const PairCoef* coef;        // class-pair coefficients (numClasses^2), or null
    int numClasses;
    int coefShared;              // the launch gives dynamic shared memory for the table: it is staged there
    const int* taskTiles;        // null: every tile is a task; else the tiles of the tasks (energies go to task slots)
    int numTasks;
};

// Bits 8..15 of a particle's flags hold its parameter class when the class tables are in use.
constexpr int kClassShift = 8;

// Every pair term of one pair.  r, invR: distance; fi, fj: flags.  Adds each term's scaled energy to e[] and returns
// the scaled dE/dr of all terms.  LEAN: the configuration has no soft core, no switching function and no order-2
// overlap, so those paths are compiled out.  UNIFORM: every particle takes part in every selected term and no pair
// is scaled (no alchemical particle, or lambda = 1), so the per-pair gate and scale tests are compiled out.
template <bool LEAN, bool UNIFORM>
__device__ __forceinline__ float pairTerms(const PairTermConfig& C, float r, float invR, const float4& a0,
                                           const float4& a1, const float4& a2, const float4& a3, int fi,
                                           const float4& b0, const float4& b1, const float4& b2, const float4& b3,
                                           int fj, bool iFirst, float e[3]) {
    float dTotal = 0.0f;
    float shared8pi = 0.0f, sharedD8pi = 0.0f, sharedR = -1.0f;
#pragma unroll
    for (int t = 0; t < 3; t++) {
        if (!((C.termMask >> t) & 1)) continue;
        if (!UNIFORM) {
            const int gate = t == 0 ? kFlagGateDisp : (t == 1 ? kFlagGateExch : kFlagGateSr);
            if (!(fi & fj & gate)) continue;
        }
        const bool alch = UNIFORM ? false : (((fi ^ fj) >> t) & 1) != 0;
        float rEff = r, invEff = invR, scR = 1.0f;
        if (!LEAN && alch && C.softShift[t] > 0.0f) {
            // r_eff = (r^6 + (1 - lambda) R^6)^(1/6), dE/dr picks up (r/r_eff)^5 (interaxPairBegin.cc, interaxPairEnd.cc)
            const float r2 = r * r;
            const float u = fmaf(r2 * r2, r2, C.softShift[t]);
            rEff = ex2Approx(lg2Approx(u) * (1.0f / 6.0f));
            invEff = rcpApprox(rEff);
            const float q = r * invEff;
            const float q2 = q * q;
            scR = q2 * q2 * q;
        }
        float E, D;
        if (t == 0) {
            dispersionEnergy(rEff, invEff, a0, b0, a1.x, b1.x, C.twoBeta, E, D);
        }
        else {
            float s8pi, ds8pi;
            if (t == 2 && C.shareOverlap && rEff == sharedR) {
                s8pi = shared8pi;
                ds8pi = sharedD8pi;
            }
            else {
                const Width Wi = t == 1 ? Width{a2.x, a3.x, a2.y, a3.y} : Width{a2.z, a3.z, a2.w, a3.w};
                const Width Wj = t == 1 ? Width{b2.x, b3.x, b2.y, b3.y} : Width{b2.z, b3.z, b2.w, b3.w};
                overlap8pi(rEff, Wi, Wj, LEAN ? 0 : C.overlapMethod[t], iFirst, s8pi, ds8pi);
                if (t == 1) {
                    shared8pi = s8pi;
                    sharedD8pi = ds8pi;
                    sharedR = rEff;
                }
            }
            if (t == 1) {
                // exchange A_i A_j S (InteraxPairTerms.h:305-312)
                const float amp = a1.y * b1.y * kInv8Pi;
                E = amp * s8pi;
                D = amp * ds8pi;
            }
            else {
                // short range (K_i+K_j)/2 St + (L_i+L_j)/2 St^2, St = 8 pi (s_i+s_j)^3 S (InteraxPairTerms.h:325-337)
                const float ws = (a2.z + b2.z) + (a3.z + b3.z);
                const float norm = ws * ws * ws;
                const float st = norm * s8pi;
                const float k = 0.5f * (a1.z + b1.z);
                const float l = 0.5f * (a1.w + b1.w);
                E = fmaf(l, st, k) * st;
                D = fmaf(2.0f * l, st, k) * norm * ds8pi;
            }
        }
        if (!LEAN) {
            D *= scR;
            if (C.useSwitch[t] && r > C.switchDist[t]) {
                const float x = (r - C.switchDist[t]) * C.invSwitchWidth[t];
                const float sv = fmaf(x * x * x, fmaf(x, fmaf(-6.0f, x, 15.0f), -10.0f), 1.0f);
                const float sd = x * x * fmaf(x, fmaf(-30.0f, x, 60.0f), -30.0f) * C.invSwitchWidth[t];
                D = fmaf(D, sv, E * sd);
                E *= sv;
            }
        }
        const float scale = alch ? C.lambda[t] : 1.0f;
        e[t] = fmaf(scale, E, e[t]);
        dTotal = fmaf(scale, D, dTotal);
    }
    return dTotal;
}

// A class-pair coefficient: through the read-only cache from the global table, or a plain load from the copy staged
// in shared memory (the read-only path cannot address shared memory).  `shared` is the same for the whole launch.
__device__ __forceinline__ float4 ldCoef(const float4* p, bool shared) { return shared ? *p : __ldg(p); }

// The same from the pair's class coefficients (see PairCoef).  Only the exact overlap method.
template <bool LEAN, bool UNIFORM>
__device__ __forceinline__ float pairTermsTable(const PairTermConfig& C, float r, float invR, const PairCoef* K,
                                                int fi, int fj, float e[3]) {
    float dTotal = 0.0f;
    float shared8pi = 0.0f, sharedD8pi = 0.0f, sharedR = -1.0f;
#pragma unroll
    for (int t = 0; t < 3; t++) {
        if (!((C.termMask >> t) & 1)) continue;
        if (!UNIFORM) {
            const int gate = t == 0 ? kFlagGateDisp : (t == 1 ? kFlagGateExch : kFlagGateSr);
            if (!(fi & fj & gate)) continue;
        }
        const bool alch = UNIFORM ? false : (((fi ^ fj) >> t) & 1) != 0;
        float rEff = r, invEff = invR, scR = 1.0f;
        if (!LEAN && alch && C.softShift[t] > 0.0f) {
            const float r2 = r * r;
            const float u = fmaf(r2 * r2, r2, C.softShift[t]);
            rEff = ex2Approx(lg2Approx(u) * (1.0f / 6.0f));
            invEff = rcpApprox(rEff);
            const float q = r * invEff;
            const float q2 = q * q;
            scR = q2 * q2 * q;
        }
        float E, D;
        if (t == 0) {
            dispersionFromCoef(rEff, invEff, ldCoef(&K->disp, C.coefShared), E, D);
        }
        else if (t == 1) {
            const float4 c = ldCoef(&K->ovC, C.coefShared);
            float s8pi, ds8pi;
            overlapFromCoef(rEff, ldCoef(&K->ovA, C.coefShared), ldCoef(&K->ovB, C.coefShared), c.x, c.y, s8pi, ds8pi);
            shared8pi = s8pi;
            sharedD8pi = ds8pi;
            sharedR = rEff;
            E = c.z * s8pi;
            D = c.z * ds8pi;
        }
        else {
            const float4 c = ldCoef(&K->srC, C.coefShared), kl = ldCoef(&K->srK, C.coefShared);
            float s8pi, ds8pi;
            if (C.shareOverlap && rEff == sharedR) {
                s8pi = shared8pi;
                ds8pi = sharedD8pi;
            }
            else overlapFromCoef(rEff, ldCoef(&K->srA, C.coefShared), ldCoef(&K->srB, C.coefShared), c.x, c.y, s8pi, ds8pi);
            const float st = c.z * s8pi;
            E = fmaf(kl.y, st, kl.x) * st;
            D = fmaf(2.0f * kl.y, st, kl.x) * c.z * ds8pi;
        }
        if (!LEAN) {
            D *= scR;
            if (C.useSwitch[t] && r > C.switchDist[t]) {
                const float x = (r - C.switchDist[t]) * C.invSwitchWidth[t];
                const float sv = fmaf(x * x * x, fmaf(x, fmaf(-6.0f, x, 15.0f), -10.0f), 1.0f);
                const float sd = x * x * fmaf(x, fmaf(-30.0f, x, 60.0f), -30.0f) * C.invSwitchWidth[t];
                D = fmaf(D, sv, E * sd);
                E *= sv;
            }
        }
        const float scale = alch ? C.lambda[t] : 1.0f;
        e[t] = fmaf(scale, E, e[t]);
        dTotal = fmaf(scale, D, dTotal);
    }
    return dTotal;
}

// Minimum image of a float-float displacement (hi, lo), c then b then a as the reference's
// ReferenceForce::getDeltaRPeriodic; the image is chosen from the float part.
__device__ __forceinline__ void minimumImageFF(float& xh, float& xl, float& yh, float& yl, float& zh, float& zl,
                                               const BoxFF& B) {
    float s = floorf(fmaf(zh, B.inv[2], 0.5f));
    xh -= s * B.c[0];
    xl -= s * B.cLo[0];
    yh -= s * B.c[1];
    yl -= s * B.cLo[1];
    zh -= s * B.c[2];
    zl -= s * B.cLo[2];
    s = floorf(fmaf(yh, B.inv[1], 0.5f));
    xh -= s * B.b[0];
    xl -= s * B.bLo[0];
    yh -= s * B.b[1];
    yl -= s * B.bLo[1];
    s = floorf(fmaf(xh, B.inv[0], 0.5f));
    xh -= s * B.a[0];
    xl -= s * B.aLo[0];
}


constexpr int kPairWarps = IX_TUNE_PAIR_WARPS;
// 1: each tile's column lists (the queue positions of each column's pairs) are built once with the queue, and the
// column forces of every round are read along them; 0: each round finds them from the row masks
constexpr int kPairColumnLists = IX_TUNE_PAIR_COLUMN_LISTS;
// 1: the column masks are always the transpose of the row masks, formed in registers (the tile list's column words
// are not read); 0: only where the rows are filtered when queued
constexpr bool kPairColumnTranspose = IX_TUNE_PAIR_COLUMN_TRANSPOSE != 0;
// 1: the class-table path without per-pair tests evaluates two queued pairs per lane at a time in packed FP32
// (computeQueuedPair2)
constexpr int kPairIlp = IX_TUNE_PAIR_ILP;
constexpr int kPairRound = IX_TUNE_PAIR_ROUND;   // queued pairs computed before their forces are gathered

// Per-warp shared memory of the pair kernel (about 6.6 KB, so that eight 4-warp blocks fit on an SM).  Parameters
// are not staged: the compute phase reads them through the read-only cache by sorted slot.  The w lanes carry what
// each pair reads besides the displacement, so that the two loads per particle bring it along: hi.w the particle's
// flags, lo.w its class-table offset (class x number of classes for an i particle, its class for a j particle), as
// integer bits.
struct PairWarpStorage {
    float4 hi[2][32];            // position offsets from the i-block center (float part); side 0 = i, 1 = j
    float4 lo[2][32];            // their float remainders
    int jslot[32];               // sorted slot of each j particle, -1 for padding
    int rowStart[32];            // queue offset of each row
    unsigned rowMask[32];
    unsigned short queue[1024];  // the tile's pairs within the cutoff, row by row: (i << 5) | j
    float4 force[kPairRound];    // force on i of each pair of the current round (j receives the opposite)
    unsigned short colList[kPairColumnLists ? 1024 : 1];   // queue positions of each column's pairs, column by column
};

__device__ __forceinline__ void stageParticle(PairWarpStorage& S, int side, int lane, int s, double cx, double cy,
                                              double cz, bool shiftImage, const PairTermConfig& C,
                                              const ListBuffers& L, const PairBuffers& P) {
    if (s >= 0) {
        double x = L.spos[3 * s] - cx, y = L.spos[3 * s + 1] - cy, z = L.spos[3 * s + 2] - cz;
        if (shiftImage) {
            // rectangular box (the shift is only enabled there)
            x -= C.box.a[0] * rint(x * C.box.inv[0]);
            y -= C.box.b[1] * rint(y * C.box.inv[1]);
            z -= C.box.c[2] * rint(z * C.box.inv[2]);
        }
        const float xh = (float)x, yh = (float)y, zh = (float)z;
        const int f = P.flags[s];
        const int cls = ((f >> kClassShift) & 0xff) * (side == 0 ? P.numClasses : 1);
        S.hi[side][lane] = make_float4(xh, yh, zh, __int_as_float(f));
        S.lo[side][lane] = make_float4((float)(x - xh), (float)(y - yh), (float)(z - zh), __int_as_float(cls));
    }
    else {
        S.hi[side][lane] = make_float4(1e30f, 1e30f, 1e30f, __int_as_float(0));
        S.lo[side][lane] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(0));
    }
    if (side == 1) S.jslot[lane] = s;
}

__device__ __forceinline__ void flushForce(const float f[3], int s, int np, long long* F) {
    if (s < 0) return;
    if (f[0] != 0.0f) atomicAddFixed(F + s, toFixed(f[0]));
    if (f[1] != 0.0f) atomicAddFixed(F + np + s, toFixed(f[1]));
    if (f[2] != 0.0f) atomicAddFixed(F + 2 * np + s, toFixed(f[2]));
}

// The displacement of j from i from their staged float-float offsets, with the per-pair minimum image where the
// staging did not place j; r2 its squared length.
__device__ __forceinline__ float pairDisplacement(const float4& hi_i, const float4& lo_i, const float4& hi_j,
                                                  const float4& lo_j, bool perPairImage, const PairTermConfig& C,
                                                  float& dx, float& dy, float& dz) {
    float dxh = hi_j.x - hi_i.x, dyh = hi_j.y - hi_i.y, dzh = hi_j.z - hi_i.z;
    float dxl = lo_j.x - lo_i.x, dyl = lo_j.y - lo_i.y, dzl = lo_j.z - lo_i.z;
    if (perPairImage) minimumImageFF(dxh, dxl, dyh, dyl, dzh, dzl, C.boxff);
    dx = dxh + dxl;
    dy = dyh + dyl;
    dz = dzh + dzl;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// Whether a pair at squared float distance r2 is within the cutoff: the float distance, and within 1e-5 of the
// cutoff the double-precision distance, as the reference decides.
__device__ __forceinline__ bool withinCutoff(float r2, const float4& hi_i, const float4& lo_i, const float4& hi_j,
                                             const float4& lo_j, bool perPairImage, const PairTermConfig& C) {
    bool inside = r2 < C.cutoff2;
    if (fabsf(r2 - C.cutoff2) < 1e-5f * C.cutoff2) {
        double ddx = ((double)hi_j.x - (double)hi_i.x) + ((double)lo_j.x - (double)lo_i.x);
        double ddy = ((double)hi_j.y - (double)hi_i.y) + ((double)lo_j.y - (double)lo_i.y);
        double ddz = ((double)hi_j.z - (double)hi_i.z) + ((double)lo_j.z - (double)lo_i.z);
        if (perPairImage) minimumImage(ddx, ddy, ddz, C.box);
        const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
        inside = sqrt(r2d) < C.cutoff;
    }
    return inside;
}

__device__ __forceinline__ bool pairInside(const float4& hi_i, const float4& lo_i, const float4& hi_j,
                                           const float4& lo_j, bool perPairImage, const PairTermConfig& C) {
    float dx, dy, dz;
    const float r2 = pairDisplacement(hi_i, lo_i, hi_j, lo_j, perPairImage, C, dx, dy, dz);
    return withinCutoff(r2, hi_i, lo_i, hi_j, lo_j, perPairImage, C);
}

// The 32 x 32 bit matrix whose row r is lane r's word, transposed (lane c receives bit r = bit c of lane r's word):
// the off-diagonal blocks of 16, 8, 4, 2 and 1 exchanged between lane pairs.
__device__ __forceinline__ unsigned transposeBits(unsigned x, int lane) {
    const unsigned masks[5] = {0x0000ffffu, 0x00ff00ffu, 0x0f0f0f0fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const int s = 16 >> k;
        const unsigned m = masks[k];
        const unsigned y = __shfl_xor_sync(0xffffffffu, x, s);
        x = (lane & s) ? ((x & ~m) | ((y & ~m) >> s)) : ((x & m) | ((y & m) << s));
    }
    return x;
}

// One queued pair: displacement, the cutoff test (CHECK: the queue holds candidates; else the pairs were filtered
// when queued), the terms.  Returns the force on i (zero outside the cutoff) and counts the pair if it interacts.
template <bool LEAN, bool TABLE, bool UNIFORM, bool CHECK>
__device__ __forceinline__ float4 computeQueuedPair(PairWarpStorage& S, int entry, int iBase, bool perPairImage,
                                                    const PairTermConfig& C, const ListBuffers& L,
                                                    const PairBuffers& P, const PairCoef* coef, float e[3],
                                                    unsigned& pairs) {
    const int i = entry >> 5, j = entry & 31;
    const float4 hi_i = S.hi[0][i], lo_i = S.lo[0][i], hi_j = S.hi[1][j], lo_j = S.lo[1][j];
    float dx, dy, dz;
    const float r2 = pairDisplacement(hi_i, lo_i, hi_j, lo_j, perPairImage, C, dx, dy, dz);
    if (CHECK && C.useCutoff && !withinCutoff(r2, hi_i, lo_i, hi_j, lo_j, perPairImage, C))
        return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const int fi = __float_as_int(hi_i.w), fj = __float_as_int(hi_j.w);
    float invR;
    const float r = sqrtRefined(r2, invR);
    float dEdR;
    if (TABLE) {
        const PairCoef* K = coef + (__float_as_int(lo_i.w) + __float_as_int(lo_j.w));
        dEdR = pairTermsTable<LEAN, UNIFORM>(C, r, invR, K, fi, fj, e);
    }
    else {
        const int si = iBase + i, sj = S.jslot[j];
        const float4 a0 = __ldg(P.p0 + si), a1 = __ldg(P.p1 + si), a2 = __ldg(P.p2 + si), a3 = __ldg(P.p3 + si);
        const float4 b0 = __ldg(P.p0 + sj), b1 = __ldg(P.p1 + sj), b2 = __ldg(P.p2 + sj), b3 = __ldg(P.p3 + sj);
        // InteraxOrder2 expands about the width of the particle with the lower original index
        const bool iFirst = LEAN ? true : __ldg(L.sortedAtom + si) < __ldg(L.sortedAtom + sj);
        dEdR = pairTerms<LEAN, UNIFORM>(C, r, invR, a0, a1, a2, a3, fi, b0, b1, b2, b3, fj, iFirst, e);
    }
    const float fs = dEdR * invR;
    pairs++;
    return make_float4(dx * fs, dy * fs, dz * fs, 0.0f);
}

// Two queued pairs of the class-table path without per-pair tests (LEAN and UNIFORM: no soft core, switch, order-2
// overlap, gate or scale), evaluated in lockstep in packed FP32 (ix_f32x2.cuh): one instruction issues each operation
// on both pairs.  A pair outside the cutoff is evaluated at its distance, where every term is finite, and masked.
// `two`: the second entry is a real pair (else the first is evaluated twice and the copy masked).  Energies
// accumulate per element in e2.
__device__ __forceinline__ void computeQueuedPair2(PairWarpStorage& S, int entry0, int entry1, bool two,
                                                   bool perPairImage, const PairTermConfig& C, const PairBuffers& P,
                                                   const PairCoef* coef, F2 (&e2)[3], unsigned& pairs,
                                                   float4& out0, float4& out1) {
    const unsigned active = __activemask();
    float dxs[2], dys[2], dzs[2], r2s[2];
    bool inside[2];
    const PairCoef* K[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const int entry = k ? entry1 : entry0;
        const int i = entry >> 5, j = entry & 31;
        const float4 hi_i = S.hi[0][i], lo_i = S.lo[0][i], hi_j = S.hi[1][j], lo_j = S.lo[1][j];
        const float r2 = pairDisplacement(hi_i, lo_i, hi_j, lo_j, perPairImage, C, dxs[k], dys[k], dzs[k]);
        const bool in = (k == 0 || two) && (!C.useCutoff || withinCutoff(r2, hi_i, lo_i, hi_j, lo_j, perPairImage, C));
        inside[k] = in;
        r2s[k] = r2;   // a pair left out is evaluated at its own (positive, finite) distance and masked
        K[k] = coef + (__float_as_int(lo_i.w) + __float_as_int(lo_j.w));
    }
    F2 invR;
    const F2 r = sqrtRefined2(f2(r2s[0], r2s[1]), invR);
    const F2 mask = f2(inside[0] ? 1.0f : 0.0f, inside[1] ? 1.0f : 0.0f);
    const F2 nmask = f2(inside[0] ? -1.0f : 0.0f, inside[1] ? -1.0f : 0.0f);
    F2 nTotal = f2(0.0f);   // -dE/dr of all terms
    if (C.termMask & 1) {
        const float4 a = ldCoef(&K[0]->disp, C.coefShared), b = ldCoef(&K[1]->disp, C.coefShared);
        F2 nE, nD;
        dispersionFromCoefP(r, invR, f2(a.x, b.x), f2(a.y, b.y), f2(a.z, b.z), f2(a.w, b.w), nE, nD);
        e2[0] = fma2(nmask, nE, e2[0]);
        nTotal = nTotal + nD;
    }
    F2 s8 = f2(0.0f), ds8 = f2(0.0f);
    if (C.termMask & 2) {
        const float4 a0 = ldCoef(&K[0]->ovA, C.coefShared), a1 = ldCoef(&K[1]->ovA, C.coefShared);
        const float4 b0 = ldCoef(&K[0]->ovB, C.coefShared), b1 = ldCoef(&K[1]->ovB, C.coefShared);
        const float4 c0 = ldCoef(&K[0]->ovC, C.coefShared), c1 = ldCoef(&K[1]->ovC, C.coefShared);
        const float4 q0 = ldCoef(&K[0]->ovQ, C.coefShared), q1 = ldCoef(&K[1]->ovQ, C.coefShared);
        const float4 u0 = ldCoef(&K[0]->ovR, C.coefShared), u1 = ldCoef(&K[1]->ovR, C.coefShared);
        overlapFromCoefP(r, f2(a0.x, a1.x), f2(b0.x, b1.x), f2(b0.y, b1.y), f2(b0.z, b1.z), f2(b0.w, b1.w),
                         f2(c0.x, c1.x), f2(c0.y, c1.y), f2(q0.x, q1.x), f2(q0.y, q1.y), f2(q0.z, q1.z),
                         f2(q0.w, q1.w), f2(u0.x, u1.x), f2(u0.y, u1.y), active, s8, ds8);
        const F2 amp = f2(c0.z, c1.z);
        e2[1] = fma2(mask, amp * s8, e2[1]);
        nTotal = fma2(amp * f2(-1.0f), ds8, nTotal);
    }
    if (C.termMask & 4) {
        const float4 c0 = ldCoef(&K[0]->srC, C.coefShared), c1 = ldCoef(&K[1]->srC, C.coefShared);
        const float4 k0 = ldCoef(&K[0]->srK, C.coefShared), k1 = ldCoef(&K[1]->srK, C.coefShared);
        if (!(C.shareOverlap && (C.termMask & 2))) {
            const float4 a0 = ldCoef(&K[0]->srA, C.coefShared), a1 = ldCoef(&K[1]->srA, C.coefShared);
            const float4 b0 = ldCoef(&K[0]->srB, C.coefShared), b1 = ldCoef(&K[1]->srB, C.coefShared);
            const float4 q0 = ldCoef(&K[0]->srQ, C.coefShared), q1 = ldCoef(&K[1]->srQ, C.coefShared);
            const float4 u0 = ldCoef(&K[0]->srR, C.coefShared), u1 = ldCoef(&K[1]->srR, C.coefShared);
            overlapFromCoefP(r, f2(a0.x, a1.x), f2(b0.x, b1.x), f2(b0.y, b1.y), f2(b0.z, b1.z), f2(b0.w, b1.w),
                             f2(c0.x, c1.x), f2(c0.y, c1.y), f2(q0.x, q1.x), f2(q0.y, q1.y), f2(q0.z, q1.z),
                             f2(q0.w, q1.w), f2(u0.x, u1.x), f2(u0.y, u1.y), active, s8, ds8);
        }
        // (K_i+K_j)/2 St + (L_i+L_j)/2 St^2, St = (s_i+s_j)^3 8 pi S
        const F2 norm = f2(c0.z, c1.z), kk = f2(k0.x, k1.x), ll = f2(k0.y, k1.y);
        const F2 st = norm * s8;
        e2[2] = fma2(mask, fma2(ll, st, kk) * st, e2[2]);
        nTotal = fma2(fma2(ll * f2(-2.0f), st, kk * f2(-1.0f)) * norm, ds8, nTotal);
    }
    const F2 fs = (nTotal * invR) * nmask;
    const F2 fx = f2(dxs[0], dxs[1]) * fs, fy = f2(dys[0], dys[1]) * fs, fz = f2(dzs[0], dzs[1]) * fs;
    out0 = make_float4(f2x(fx), f2x(fy), f2x(fz), 0.0f);
    out1 = make_float4(f2y(fx), f2y(fy), f2y(fz), 0.0f);
    pairs += (unsigned)inside[0] + (unsigned)inside[1];
}

template <bool LEAN, bool TABLE, bool UNIFORM = false>
__global__ void __launch_bounds__(32 * kPairWarps, IX_TUNE_PAIR_MIN_BLOCKS) kPairTiles(ListBuffers L, PairBuffers P, PairTermConfig C) {
    __shared__ PairWarpStorage storage[kPairWarps];
    extern __shared__ float4 pairShared[];
    // the candidates are filtered against the cutoff when queued, except on the class-table path without soft core,
    // switch or order-2 overlap, whose pairs are cheap enough that the filter costs what it saves: there the compute
    // phase tests each candidate
    constexpr bool PREFILTER = !(LEAN && TABLE);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    PairWarpStorage& S = storage[warp];
    // the class-pair table, staged in shared memory when the launch gives room for it
    const PairCoef* coef = P.coef;
    if (TABLE && P.coefShared) {
        const int words = P.numClasses * P.numClasses * (int)(sizeof(PairCoef) / sizeof(float4));
        const float4* src = reinterpret_cast<const float4*>(P.coef);
        for (int k = threadIdx.x; k < words; k += blockDim.x) pairShared[k] = __ldg(src + k);
        __syncthreads();
        coef = reinterpret_cast<const PairCoef*>(pairShared);
    }
    const int numTasks = P.taskTiles ? P.numTasks : min(*L.numTiles, L.tileCap);
    const unsigned ltMask = laneMaskLt();
    unsigned long long pairs = 0;
    for (;;) {
        int task = 0;
        if (lane == 0) task = atomicAdd(L.taskCounter, 1);
        task = __shfl_sync(0xffffffffu, task, 0);
        if (task >= numTasks) break;
        const int t = P.taskTiles ? P.taskTiles[task] : (L.tileOrder ? L.tileOrder[task] : task);
        const int I = L.tileIBlock[t];
        const int iBase = I * 32;
        const float4 center = L.bbox[2 * I];
        const bool shiftImage = C.periodic && center.w != 0.0f;
        const bool perPairImage = C.periodic && !shiftImage;
        const double cx = center.x, cy = center.y, cz = center.z;
        float fi[3] = {0.0f, 0.0f, 0.0f};
        {
            const int jslot = L.tileJ[32 * t + lane];
            unsigned row = L.tileMask[64 * t + lane];
            unsigned column = (PREFILTER || kPairColumnTranspose) ? 0u : L.tileMask[64 * t + 32 + lane];
            __syncwarp();
            stageParticle(S, 0, lane, iBase + lane, cx, cy, cz, false, C, L, P);
            stageParticle(S, 1, lane, jslot, cx, cy, cz, shiftImage, C, L, P);
            if (C.alchOnlyBit) {
                // keep the pairs with exactly one alchemical particle
                const bool ia = (__float_as_int(S.hi[0][lane].w) & C.alchOnlyBit) != 0;
                const bool ja = (__float_as_int(S.hi[1][lane].w) & C.alchOnlyBit) != 0;
                const unsigned iAlch = __ballot_sync(0xffffffffu, ia), jAlch = __ballot_sync(0xffffffffu, ja);
                row &= ia ? ~jAlch : jAlch;
                column &= ja ? ~iAlch : iAlch;
            }
            __syncwarp();
            if (PREFILTER && C.useCutoff) {
                // the row's candidates within the cutoff at the current positions
                const float4 hi_i = S.hi[0][lane], lo_i = S.lo[0][lane];
                unsigned kept = 0;
                for (unsigned m = row; m; m &= m - 1) {
                    const int j = __ffs(m) - 1;
                    if (pairInside(hi_i, lo_i, S.hi[1][j], S.lo[1][j], perPairImage, C)) kept |= 1u << j;
                }
                row = kept;
            }
            // the filtered columns are the transpose of the filtered rows; unfiltered, the list holds them (or, with
            // kPairColumnTranspose, they are formed here the same way)
            if (PREFILTER || kPairColumnTranspose) column = transposeBits(row, lane);
            // queue the kept pairs row by row
            const int count = __popc(row);
            int start = count;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, start, o);
                if (lane >= o) start += v;
            }
            const int total = __shfl_sync(0xffffffffu, start, 31);
            start -= count;
            S.rowStart[lane] = start;
            S.rowMask[lane] = row;
            for (unsigned m = row, q = start; m; m &= m - 1, q++)
                S.queue[q] = (unsigned short)((lane << 5) | (__ffs(m) - 1));
            __syncwarp();
            // column lists: for each row i of this lane's column, the position of (i, lane) in the queue (rising)
            int colPtr = 0, colEnd = 0;
            if (kPairColumnLists) {
                const int ccount = __popc(column);
                int cstart = ccount;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, cstart, o);
                    if (lane >= o) cstart += v;
                }
                cstart -= ccount;
                colPtr = cstart;
                colEnd = cstart + ccount;
                for (unsigned m = column, q = cstart; m; m &= m - 1, q++) {
                    const int i = __ffs(m) - 1;
                    S.colList[q] = (unsigned short)(S.rowStart[i] + __popc(S.rowMask[i] & ltMask));
                }
                __syncwarp();
            }
            float e[3] = {0.0f, 0.0f, 0.0f};
            F2 e2[3] = {f2(0.0f), f2(0.0f), f2(0.0f)};   // the packed path's energies, per element
            float fj[3] = {0.0f, 0.0f, 0.0f};
            unsigned tilePairs = 0;
            for (int base = 0; base < total; base += kPairRound) {
                const int n = min(kPairRound, total - base);
                if (kPairIlp && LEAN && TABLE && UNIFORM) {
                    // two pairs per lane at a time: p and p + 32
                    for (int p = lane; p < n; p += 64) {
                        const bool two = p + 32 < n;
                        float4 f0, f1;
                        computeQueuedPair2(S, S.queue[base + p], S.queue[base + (two ? p + 32 : p)], two,
                                           perPairImage, C, P, coef, e2, tilePairs, f0, f1);
                        S.force[p] = f0;
                        if (two) S.force[p + 32] = f1;
                    }
                }
                else
                    for (int p = lane; p < n; p += 32)
                        S.force[p] = computeQueuedPair<LEAN, TABLE, UNIFORM, !PREFILTER>(
                            S, S.queue[base + p], iBase, perPairImage, C, L, P, coef, e, tilePairs);
                __syncwarp();
                // i side: this lane's row, contiguous in the queue
                const int a = max(start, base), b = min(start + count, base + n);
                for (int q = a; q < b; q++) {
                    const float4 f = S.force[q - base];
                    fi[0] += f.x;
                    fi[1] += f.y;
                    fi[2] += f.z;
                }
                if (kPairColumnLists) {
                    // j side: along this lane's column list, the positions inside this round
                    for (; colPtr < colEnd; colPtr++) {
                        const int q = S.colList[colPtr] - base;
                        if (q >= n) break;
                        const float4 f = S.force[q];
                        fj[0] -= f.x;
                        fj[1] -= f.y;
                        fj[2] -= f.z;
                    }
                }
                else {
                    // j side: the pair (i, lane) of each row i of this round that holds it
                    unsigned rows = column & __ballot_sync(0xffffffffu, start < base + n && start + count > base);
                    while (rows) {
                        const int i = __ffs(rows) - 1;
                        rows &= rows - 1;
                        const int q = S.rowStart[i] + __popc(S.rowMask[i] & ltMask) - base;
                        if (q >= 0 && q < n) {
                            const float4 f = S.force[q];
                            fj[0] -= f.x;
                            fj[1] -= f.y;
                            fj[2] -= f.z;
                        }
                    }
                }
                __syncwarp();
            }
            pairs += tilePairs;
            if (kPairIlp && LEAN && TABLE && UNIFORM)
                for (int k = 0; k < 3; k++) e[k] = f2x(e2[k]) + f2y(e2[k]);
            flushForce(fj, jslot, L.np, P.forceFixed);
            // the tile's energies: a fixed reduction tree over the lanes, one slot per tile
            for (int k = 0; k < 3; k++) {
                const double sum = warpSumD((double)e[k]);
                if (lane == 0) P.taskEnergy[3 * (P.taskTiles ? task : t) + k] = sum;
            }
        }
        flushForce(fi, iBase + lane, L.np, P.forceFixed);
    }
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if (lane == 0 && pairs) atomicAdd(P.pairCount, pairs);
}

}  // namespace ix
