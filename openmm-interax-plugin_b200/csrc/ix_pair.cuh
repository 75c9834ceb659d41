// Fused pair kernel: the dispersion, exchange and short-range terms of every interacting pair in one pass over the
// tile list (the reference runs them as snippets of OpenMM's nonbonded kernel in one pass,
// platforms/common/src/CommonInteraxKernels.cpp:139-219, kernels interaxPairBegin.cc / interaxPairEnd.cc).
//
// Warps take tiles from a counter in global memory until none is left (dynamic balance).  Per tile:
//   1. staging: the 32 i particles and the tile's 32 j particles are written to shared memory as
//      float-float offsets from the i-block's center (the double-precision difference split into a float and its
//      float remainder).  In large rectangular boxes each j particle is placed at its minimum image relative to the
//      block center here, once, instead of per pair;
//   2. queue: the tile's row masks (built with the list) give the candidate pairs; each lane writes its row's pairs
//      to a per-warp queue at the row's offset (a warp prefix sum of the row counts), so that the expensive phase
//      runs with every lane busy and no per-step candidate test;
//   3. compute phase, in rounds of kPairRound queued pairs: each lane takes one pair, forms the displacement as
//      (xj - xi) + (lo_j - lo_i) (the precision of the double difference, without double arithmetic), applies the
//      exact cutoff test (borderline cases decided in double), evaluates the three terms in float and stores the
//      pair force in shared memory;
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
// 1: the class-table path without per-pair tests evaluates two queued pairs per lane at a time (computeQueuedPair2)
constexpr int kPairIlp = IX_TUNE_PAIR_ILP;
constexpr int kPairRound = IX_TUNE_PAIR_ROUND;   // queued pairs computed before their forces are gathered

// Per-warp shared memory of the pair kernel (about 6.8 KB, so that eight 4-warp blocks fit on an SM).  Parameters
// are not staged: the compute phase reads them through the read-only cache by sorted slot.
struct PairWarpStorage {
    float4 hi[2][32];            // position offsets from the i-block center (float part); side 0 = i, 1 = j
    float4 lo[2][32];            // their float remainders
    int flags[2][32];
    int jslot[32];               // sorted slot of each j particle, -1 for padding
    int rowStart[32];            // queue offset of each row
    unsigned rowMask[32];
    unsigned short queue[1024];  // the tile's candidate pairs, row by row: (i << 5) | j
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
        S.hi[side][lane] = make_float4(xh, yh, zh, 0.0f);
        S.lo[side][lane] = make_float4((float)(x - xh), (float)(y - yh), (float)(z - zh), 0.0f);
        S.flags[side][lane] = P.flags[s];
    }
    else {
        S.flags[side][lane] = 0;
        S.hi[side][lane] = make_float4(1e30f, 1e30f, 1e30f, 0.0f);
        S.lo[side][lane] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (side == 1) S.jslot[lane] = s;
}

__device__ __forceinline__ void flushForce(const float f[3], int s, int np, long long* F) {
    if (s < 0) return;
    if (f[0] != 0.0f) atomicAddFixed(F + s, toFixed(f[0]));
    if (f[1] != 0.0f) atomicAddFixed(F + np + s, toFixed(f[1]));
    if (f[2] != 0.0f) atomicAddFixed(F + 2 * np + s, toFixed(f[2]));
}

// One queued pair: displacement, exact cutoff test, the terms.  Returns the force on i (zero outside the cutoff).
template <bool LEAN, bool TABLE, bool UNIFORM>
__device__ __forceinline__ float4 computeQueuedPair(PairWarpStorage& S, int entry, int iBase, bool perPairImage,
                                                    const PairTermConfig& C, const ListBuffers& L,
                                                    const PairBuffers& P, const PairCoef* coef, float e[3],
                                                    unsigned& pairs) {
    const int i = entry >> 5, j = entry & 31;
    const float4 hi_i = S.hi[0][i], hi_j = S.hi[1][j], lo_i = S.lo[0][i], lo_j = S.lo[1][j];
    float dxh = hi_j.x - hi_i.x, dyh = hi_j.y - hi_i.y, dzh = hi_j.z - hi_i.z;
    float dxl = lo_j.x - lo_i.x, dyl = lo_j.y - lo_i.y, dzl = lo_j.z - lo_i.z;
    if (perPairImage) minimumImageFF(dxh, dxl, dyh, dyl, dzh, dzl, C.boxff);
    const float dx = dxh + dxl, dy = dyh + dyl, dz = dzh + dzl;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    bool inside = true;
    if (C.useCutoff) {
        inside = r2 < C.cutoff2;
        if (fabsf(r2 - C.cutoff2) < 1e-5f * C.cutoff2) {
            // decide as the reference does, on the double precision distance
            double ddx = ((double)hi_j.x - (double)hi_i.x) + ((double)lo_j.x - (double)lo_i.x);
            double ddy = ((double)hi_j.y - (double)hi_i.y) + ((double)lo_j.y - (double)lo_i.y);
            double ddz = ((double)hi_j.z - (double)hi_i.z) + ((double)lo_j.z - (double)lo_i.z);
            if (perPairImage) minimumImage(ddx, ddy, ddz, C.box);
            const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
            inside = sqrt(r2d) < C.cutoff;
        }
    }
    const int fi = S.flags[0][i], fj = S.flags[1][j];
    if (!inside) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float invR;
    const float r = sqrtRefined(r2, invR);
    float dEdR;
    if (TABLE) {
        const int ci = (fi >> kClassShift) & 0xff, cj = (fj >> kClassShift) & 0xff;
        dEdR = pairTermsTable<LEAN, UNIFORM>(C, r, invR, coef + ci * P.numClasses + cj, fi, fj, e);
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
// overlap, gate or scale), their arithmetic in one straight sequence so that each lane keeps two independent chains in
// flight; a pair outside the cutoff is evaluated at a harmless distance and masked.  The results are those of
// computeQueuedPair, operation for operation.  `two`: the second entry is a real pair.
__device__ __forceinline__ void computeQueuedPair2(PairWarpStorage& S, int entry0, int entry1, bool two,
                                                   bool perPairImage, const PairTermConfig& C, const PairBuffers& P,
                                                   const PairCoef* coef, float e[3], unsigned& pairs,
                                                   float4& out0, float4& out1) {
    const int entry[2] = {entry0, entry1};
    float dx[2], dy[2], dz[2], r[2], invR[2];
    bool inside[2];
    const PairCoef* K[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const int i = entry[k] >> 5, j = entry[k] & 31;
        const float4 hi_i = S.hi[0][i], hi_j = S.hi[1][j], lo_i = S.lo[0][i], lo_j = S.lo[1][j];
        float dxh = hi_j.x - hi_i.x, dyh = hi_j.y - hi_i.y, dzh = hi_j.z - hi_i.z;
        float dxl = lo_j.x - lo_i.x, dyl = lo_j.y - lo_i.y, dzl = lo_j.z - lo_i.z;
        if (perPairImage) minimumImageFF(dxh, dxl, dyh, dyl, dzh, dzl, C.boxff);
        dx[k] = dxh + dxl;
        dy[k] = dyh + dyl;
        dz[k] = dzh + dzl;
        const float r2 = fmaf(dx[k], dx[k], fmaf(dy[k], dy[k], dz[k] * dz[k]));
        bool in = k == 0 || two;
        if (C.useCutoff) {
            bool within = r2 < C.cutoff2;
            if (fabsf(r2 - C.cutoff2) < 1e-5f * C.cutoff2) {
                double ddx = ((double)hi_j.x - (double)hi_i.x) + ((double)lo_j.x - (double)lo_i.x);
                double ddy = ((double)hi_j.y - (double)hi_i.y) + ((double)lo_j.y - (double)lo_i.y);
                double ddz = ((double)hi_j.z - (double)hi_i.z) + ((double)lo_j.z - (double)lo_i.z);
                if (perPairImage) minimumImage(ddx, ddy, ddz, C.box);
                const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
                within = sqrt(r2d) < C.cutoff;
            }
            in = in && within;
        }
        inside[k] = in;
        // a pair left out is evaluated at half the cutoff, where every term is finite, and its results dropped
        r[k] = sqrtRefined(in ? r2 : 0.25f * C.cutoff2, invR[k]);
        const int fi = S.flags[0][i], fj = S.flags[1][j];
        const int ci = (fi >> kClassShift) & 0xff, cj = (fj >> kClassShift) & 0xff;
        K[k] = coef + ci * P.numClasses + cj;
    }
    float dTotal[2] = {0.0f, 0.0f};
    float s8[2] = {0.0f, 0.0f}, ds8[2] = {0.0f, 0.0f};
    if (C.termMask & 1) {
        const float4 kd[2] = {ldCoef(&K[0]->disp, C.coefShared), ldCoef(&K[1]->disp, C.coefShared)};
        float E[2], D[2];
        dispersionFromCoef2(r, invR, kd, E, D);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            e[0] += inside[k] ? E[k] : 0.0f;
            dTotal[k] += D[k];
        }
    }
    if (C.termMask & 2) {
        const float4 a[2] = {ldCoef(&K[0]->ovA, C.coefShared), ldCoef(&K[1]->ovA, C.coefShared)};
        const float4 b[2] = {ldCoef(&K[0]->ovB, C.coefShared), ldCoef(&K[1]->ovB, C.coefShared)};
        const float4 c[2] = {ldCoef(&K[0]->ovC, C.coefShared), ldCoef(&K[1]->ovC, C.coefShared)};
        const float k1[2] = {c[0].x, c[1].x}, k2[2] = {c[0].y, c[1].y};
        overlapFromCoef2(r, a, b, k1, k2, s8, ds8);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            e[1] += inside[k] ? c[k].z * s8[k] : 0.0f;
            dTotal[k] = fmaf(1.0f, c[k].z * ds8[k], dTotal[k]);
        }
    }
    if (C.termMask & 4) {
        const float4 c[2] = {ldCoef(&K[0]->srC, C.coefShared), ldCoef(&K[1]->srC, C.coefShared)};
        const float4 kl[2] = {ldCoef(&K[0]->srK, C.coefShared), ldCoef(&K[1]->srK, C.coefShared)};
        if (!(C.shareOverlap && (C.termMask & 2))) {
            const float4 a[2] = {ldCoef(&K[0]->srA, C.coefShared), ldCoef(&K[1]->srA, C.coefShared)};
            const float4 b[2] = {ldCoef(&K[0]->srB, C.coefShared), ldCoef(&K[1]->srB, C.coefShared)};
            const float k1[2] = {c[0].x, c[1].x}, k2[2] = {c[0].y, c[1].y};
            overlapFromCoef2(r, a, b, k1, k2, s8, ds8);
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const float st = c[k].z * s8[k];
            const float E = fmaf(kl[k].y, st, kl[k].x) * st;
            const float D = fmaf(2.0f * kl[k].y, st, kl[k].x) * c[k].z * ds8[k];
            e[2] += inside[k] ? E : 0.0f;
            dTotal[k] += D;
        }
    }
    float4 out[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float fs = inside[k] ? dTotal[k] * invR[k] : 0.0f;
        out[k] = make_float4(dx[k] * fs, dy[k] * fs, dz[k] * fs, 0.0f);
        pairs += inside[k];
    }
    out0 = out[0];
    out1 = out[1];
}

template <bool LEAN, bool TABLE, bool UNIFORM = false>
__global__ void __launch_bounds__(32 * kPairWarps, IX_TUNE_PAIR_MIN_BLOCKS) kPairTiles(ListBuffers L, PairBuffers P, PairTermConfig C) {
    __shared__ PairWarpStorage storage[kPairWarps];
    extern __shared__ float4 pairShared[];
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
            unsigned column = L.tileMask[64 * t + 32 + lane];
            __syncwarp();
            stageParticle(S, 0, lane, iBase + lane, cx, cy, cz, false, C, L, P);
            stageParticle(S, 1, lane, jslot, cx, cy, cz, shiftImage, C, L, P);
            if (C.alchOnlyBit) {
                // keep the pairs with exactly one alchemical particle
                const bool ia = (S.flags[0][lane] & C.alchOnlyBit) != 0, ja = (S.flags[1][lane] & C.alchOnlyBit) != 0;
                const unsigned iAlch = __ballot_sync(0xffffffffu, ia), jAlch = __ballot_sync(0xffffffffu, ja);
                row &= ia ? ~jAlch : jAlch;
                column &= ja ? ~iAlch : iAlch;
            }
            // queue the tile's candidate pairs row by row
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
                                           perPairImage, C, P, coef, e, tilePairs, f0, f1);
                        S.force[p] = f0;
                        if (two) S.force[p + 32] = f1;
                    }
                }
                else
                    for (int p = lane; p < n; p += 32)
                        S.force[p] = computeQueuedPair<LEAN, TABLE, UNIFORM>(S, S.queue[base + p], iBase,
                                                                              perPairImage, C, L, P, coef, e,
                                                                              tilePairs);
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
