// Fused pair kernel: the dispersion, exchange and short-range terms of every interacting pair in one pass over the
// tile list (the reference runs them as snippets of OpenMM's nonbonded kernel in one pass,
// platforms/common/src/CommonInteraxKernels.cpp:139-219, kernels interaxPairBegin.cc / interaxPairEnd.cc).
//
// One warp processes one task (up to kTaskTiles tiles of the same i-block).  Per tile:
//   1. the 32 i and 32 j particles are staged in shared memory (double positions, float parameters);
//   2. test phase: the 32 x 32 pairs are tested in rotation order (lane l, rotation k pairs i = l with slot
//      j = (l + k) mod 32) with float positions and a small margin, and the candidates are compacted into a
//      per-warp queue with ballots, so that the expensive phase runs with every lane busy;
//   3. compute phase: each lane takes one queued pair, forms the displacement in double precision (minimum image in
//      double), applies the exact cutoff test, evaluates the three terms in float and accumulates the pair force on
//      i and j in shared memory;
//   4. the j forces are added to the global 64-bit fixed-point force buffer (scale 2^32); the i forces once per task.
// Energies accumulate per lane in double and are added in fixed point, so the result does not depend on the order in
// which warps run.
#pragma once

#include "ix_nblist.cuh"
#include "ix_pair_math.cuh"

namespace ix {

// Particle flags in the sorted parameter arrays.
constexpr int kFlagReal = 1 << 3;
constexpr int kFlagGateDisp = 1 << 4;    // alpha != 0
constexpr int kFlagGateExch = 1 << 5;    // exchange width != 0
constexpr int kFlagGateSr = 1 << 6;      // short-range width != 0

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
    float cutoff2, testCutoff2;
    double cutoff;
    Box box;
    BoxF boxf;
};

struct PairBuffers {
    const float4* p0;            // sorted: m1, m2, m3, alpha
    const float4* p1;            // sorted: dispersion width, amplitude A, K, L
    const float4* p2;            // sorted: exchange width, 1/width, short-range width, 1/width
    const float4* p3;            // sorted: the float remainders of p2's four values (float-float widths)
    const int* flags;            // sorted
    long long* forceFixed;       // 3 x np, sorted order, SoA
    double* energyPartials;      // 3 per warp of the grid, summed in a fixed order afterwards
    unsigned long long* pairCount;
};

// Every pair term of one pair.  r, invR: distance; fi, fj: flags.  Adds each term's scaled energy to e[] and returns
// the scaled dE/dr of all terms.
__device__ __forceinline__ float pairTerms(const PairTermConfig& C, float r, float invR, float4 a0, float4 a1,
                                           float4 a2, float4 a3, int fi, float4 b0, float4 b1, float4 b2,
                                           float4 b3, int fj, bool iFirst, float e[3]) {
    float dTotal = 0.0f;
    float shared8pi = 0.0f, sharedD8pi = 0.0f, sharedR = -1.0f;
#pragma unroll
    for (int t = 0; t < 3; t++) {
        if (!((C.termMask >> t) & 1)) continue;
        const int gate = t == 0 ? kFlagGateDisp : (t == 1 ? kFlagGateExch : kFlagGateSr);
        if (!(fi & fj & gate)) continue;
        const bool alch = ((fi ^ fj) >> t) & 1;
        float rEff = r, invEff = invR, scR = 1.0f;
        if (alch && C.softShift[t] > 0.0f) {
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
            else if (t == 1) {
                overlap8pi(rEff, Width{a2.x, a3.x, a2.y, a3.y}, Width{b2.x, b3.x, b2.y, b3.y}, C.overlapMethod[1],
                           iFirst, s8pi, ds8pi);
                shared8pi = s8pi;
                sharedD8pi = ds8pi;
                sharedR = rEff;
            }
            else {
                overlap8pi(rEff, Width{a2.z, a3.z, a2.w, a3.w}, Width{b2.z, b3.z, b2.w, b3.w}, C.overlapMethod[2],
                           iFirst, s8pi, ds8pi);
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
        D *= scR;
        if (C.useSwitch[t] && r > C.switchDist[t]) {
            const float x = (r - C.switchDist[t]) * C.invSwitchWidth[t];
            const float sv = fmaf(x * x * x, fmaf(x, fmaf(-6.0f, x, 15.0f), -10.0f), 1.0f);
            const float sd = x * x * fmaf(x, fmaf(-30.0f, x, 60.0f), -30.0f) * C.invSwitchWidth[t];
            D = fmaf(D, sv, E * sd);
            E *= sv;
        }
        const float scale = alch ? C.lambda[t] : 1.0f;
        e[t] = fmaf(scale, E, e[t]);
        dTotal = fmaf(scale, D, dTotal);
    }
    return dTotal;
}

struct PairWarpStorage {
    double x[2][32], y[2][32], z[2][32];
    float4 pf[2][32];
    float4 a0[2][32], a1[2][32], a2[2][32], a3[2][32];
    int flags[2][32], orig[2][32], slot[2][32];
    float fx[2][32], fy[2][32], fz[2][32];
    unsigned short queue[1024];
};

constexpr int kPairWarps = 4;

__device__ __forceinline__ void stageParticle(PairWarpStorage& S, int side, int lane, int s, const ListBuffers& L,
                                              const PairBuffers& P) {
    if (s >= 0) {
        S.x[side][lane] = L.spos[3 * s];
        S.y[side][lane] = L.spos[3 * s + 1];
        S.z[side][lane] = L.spos[3 * s + 2];
        S.pf[side][lane] = L.sposf[s];
        S.a0[side][lane] = P.p0[s];
        S.a1[side][lane] = P.p1[s];
        S.a2[side][lane] = P.p2[s];
        S.a3[side][lane] = P.p3[s];
        S.flags[side][lane] = P.flags[s];
        S.orig[side][lane] = L.sortedAtom[s];
        S.slot[side][lane] = s;
    }
    else {
        S.flags[side][lane] = 0;
        S.orig[side][lane] = -1;
        S.slot[side][lane] = -1;
        S.pf[side][lane] = make_float4(1e30f, 1e30f, 1e30f, 0.0f);
    }
    S.fx[side][lane] = 0.0f;
    S.fy[side][lane] = 0.0f;
    S.fz[side][lane] = 0.0f;
}

__device__ __forceinline__ void flushForce(const PairWarpStorage& S, int side, int lane, int np, long long* F) {
    const int s = S.slot[side][lane];
    if (s < 0) return;
    const float fx = S.fx[side][lane], fy = S.fy[side][lane], fz = S.fz[side][lane];
    if (fx != 0.0f) atomicAddFixed(F + s, toFixed(fx));
    if (fy != 0.0f) atomicAddFixed(F + np + s, toFixed(fy));
    if (fz != 0.0f) atomicAddFixed(F + 2 * np + s, toFixed(fz));
}

__global__ void __launch_bounds__(32 * kPairWarps) kPairTiles(ListBuffers L, PairBuffers P, PairTermConfig C) {
    __shared__ PairWarpStorage storage[kPairWarps];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    PairWarpStorage& S = storage[warp];
    const int numTasks = min(*L.numTasks, L.taskCap);
    double eAcc[3] = {0.0, 0.0, 0.0};
    unsigned long long pairs = 0;
    for (int task = blockIdx.x * kPairWarps + warp; task < numTasks; task += gridDim.x * kPairWarps) {
        const int2 tk = L.tasks[task];
        const int I = L.tileIBlock[tk.x];
        __syncwarp();
        stageParticle(S, 0, lane, I * 32 + lane, L, P);
        for (int t = tk.x; t < tk.x + tk.y; t++) {
            const int jslot = L.tileJ[32 * t + lane];
            const int ex = L.tileExcl[t];
            const unsigned excl = ex >= 0 ? L.exclMasks[32 * ex + lane] : 0u;
            __syncwarp();
            stageParticle(S, 1, lane, jslot, L, P);
            __syncwarp();
            // test phase
            const float4 xi = S.pf[0][lane];
            const int si = S.slot[0][lane];
            const int fiTest = S.flags[0][lane];
            int qn = 0;
#pragma unroll 4
            for (int k = 0; k < 32; k++) {
                const int jj = (lane + k) & 31;
                const float4 xj = S.pf[1][jj];
                bool valid = (fiTest & S.flags[1][jj] & kFlagReal) && S.slot[1][jj] > si && !((excl >> jj) & 1u);
                if (C.useCutoff) {
                    float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
                    if (C.periodic) minimumImageF(dx, dy, dz, C.boxf);
                    valid = valid && fmaf(dx, dx, fmaf(dy, dy, dz * dz)) < C.testCutoff2;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, valid);
                if (valid) S.queue[qn + __popc(bal & laneMaskLt())] = (unsigned short)((lane << 5) | jj);
                qn += __popc(bal);
            }
            __syncwarp();
            // compute phase
            float e[3] = {0.0f, 0.0f, 0.0f};
            for (int q = 0; q < qn; q += 32) {
                if (q + lane < qn) {
                    const int entry = S.queue[q + lane];
                    const int i = entry >> 5, j = entry & 31;
                    double dxd = S.x[1][j] - S.x[0][i];
                    double dyd = S.y[1][j] - S.y[0][i];
                    double dzd = S.z[1][j] - S.z[0][i];
                    if (C.periodic) minimumImage(dxd, dyd, dzd, C.box);
                    const float dx = (float)dxd, dy = (float)dyd, dz = (float)dzd;
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    bool inside = true;
                    if (C.useCutoff) {
                        inside = r2 < C.cutoff2;
                        if (fabsf(r2 - C.cutoff2) < 1e-5f * C.cutoff2) {
                            // decide as the reference does, on the double precision distance
                            const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(dxd, dxd), __dmul_rn(dyd, dyd)),
                                                         __dmul_rn(dzd, dzd));
                            inside = sqrt(r2d) < C.cutoff;
                        }
                    }
                    const int fi = S.flags[0][i], fj = S.flags[1][j];
                    if (inside && (fi & fj & (kFlagGateDisp | kFlagGateExch | kFlagGateSr))) {
                        float invR;
                        const float r = sqrtRefined(r2, invR);
                        const float dEdR = pairTerms(C, r, invR, S.a0[0][i], S.a1[0][i], S.a2[0][i], S.a3[0][i],
                                                     fi, S.a0[1][j], S.a1[1][j], S.a2[1][j], S.a3[1][j], fj,
                                                     S.orig[0][i] < S.orig[1][j], e);
                        const float fs = dEdR * invR;
                        const float fxv = dx * fs, fyv = dy * fs, fzv = dz * fs;
                        atomicAdd(&S.fx[0][i], fxv);
                        atomicAdd(&S.fy[0][i], fyv);
                        atomicAdd(&S.fz[0][i], fzv);
                        atomicAdd(&S.fx[1][j], -fxv);
                        atomicAdd(&S.fy[1][j], -fyv);
                        atomicAdd(&S.fz[1][j], -fzv);
                        pairs++;
                    }
                }
            }
            eAcc[0] += e[0];
            eAcc[1] += e[1];
            eAcc[2] += e[2];
            __syncwarp();
            flushForce(S, 1, lane, L.np, P.forceFixed);
        }
        __syncwarp();
        flushForce(S, 0, lane, L.np, P.forceFixed);
    }
    // each warp's energy, in a fixed order of its tasks and a fixed reduction tree; the partials of all warps are
    // summed in a fixed order by kReduceEnergies, so the total is the same on every run
    const int globalWarp = blockIdx.x * kPairWarps + warp;
    for (int t = 0; t < 3; t++) {
        const double sum = warpSumD(eAcc[t]);
        if (lane == 0) P.energyPartials[3 * globalWarp + t] = sum;
    }
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if (lane == 0 && pairs) atomicAdd(P.pairCount, pairs);
}

}  // namespace ix
