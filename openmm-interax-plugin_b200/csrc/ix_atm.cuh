// Axilrod-Teller-Muto three-body kernels (the reference's five-kernel pipeline is
// platforms/common/src/kernels/interaxThreeBody.cc:11-655 with host code CommonInteraxKernels.cpp:386-646; the FP64
// definition is openmmapi/include/internal/InteraxThreeBodyTerms.h:51-146 and
// platforms/reference/src/ReferenceInteraxThreeBodyIxn.cpp:84-135).
//
//   kSiteCentroids       site positions (unweighted centroids, double) and the site rebuild check
//   kSiteNeighbors       (rebuild only) per site A the sites B > A of other molecules within cutoff + skin
//   kTriples             one warp per site A: the neighbors within the cutoff are staged in shared memory with their
//                        double-precision minimum-image displacements from A; the pairs (B, C) of them are
//                        enumerated by a flat triangular index so that all lanes are busy; each triple is counted
//                        once (A lowest), evaluated in float, and its forces on B and C accumulate in shared memory
//   kSpreadSiteForces    the site forces, shared equally among each site's particles, into the particle forces
#pragma once

#include "ix_common.cuh"

namespace ix {

constexpr float kSiteSkin = 0.1f;

struct AtmConfig {
    int numSites;
    int periodic;
    Box box;
    BoxF boxf;
    float cutoff2;
    float listCutoff2;
    float scale;                 // scale factor
    float lambda;                // alchemical parameter (1 without alchemical sites)
    int useTangToennies;
    float twoBeta;               // 2 x damping scale
    float invCentroidRadius;     // 0 = no centroid damping
    float maxMove2;
};

struct AtmBuffers {
    const int* siteOffsets;      // numSites + 1
    const int* siteParticles;
    const float4* siteParams;    // alpha, frequency, width, alchemical (0/1)
    const int* molecule;         // effective molecule (negative input already replaced by -1 - site)
    double* sitePos;             // numSites x 3
    double* siteRef;             // numSites x 3, at the last list build
    int* flag;                   // [0] rebuild, [1] neighbor overflow
    int* nbrCount;               // numSites
    int* nbr;                    // numSites x cap
    int cap;
    long long* siteForce;        // 3 x numSites, SoA fixed point
    long long* particleForce;    // 3 x numParticles, SoA fixed point (original order)
    int numParticles;
    double* energyPartials;      // one per warp of the triple kernel's grid
    unsigned long long* tripleCount;
};

__global__ void kSiteCentroids(AtmBuffers A, AtmConfig C, const double* pos) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    if (s < C.numSites) {
        double c[3] = {0.0, 0.0, 0.0};
        const int b = A.siteOffsets[s], e = A.siteOffsets[s + 1];
        for (int k = b; k < e; k++) {
            const int p = A.siteParticles[k];
            c[0] += pos[3 * p];
            c[1] += pos[3 * p + 1];
            c[2] += pos[3 * p + 2];
        }
        const double n = (double)(e - b);
        for (int d = 0; d < 3; d++) {
            c[d] /= n;
            A.sitePos[3 * s + d] = c[d];
        }
        const double dx = c[0] - A.siteRef[3 * s], dy = c[1] - A.siteRef[3 * s + 1], dz = c[2] - A.siteRef[3 * s + 2];
        moved = (float)(dx * dx + dy * dy + dz * dz) > C.maxMove2;
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) atomicOr(A.flag, 1);
}

__device__ __forceinline__ void siteDelta(const AtmBuffers& A, const AtmConfig& C, int from, int to, double d[3]) {
    d[0] = A.sitePos[3 * to] - A.sitePos[3 * from];
    d[1] = A.sitePos[3 * to + 1] - A.sitePos[3 * from + 1];
    d[2] = A.sitePos[3 * to + 2] - A.sitePos[3 * from + 2];
    if (C.periodic) minimumImage(d[0], d[1], d[2], C.box);
}

// One warp per site A scans the sites above it.  The list is in increasing site order.
__global__ void kSiteNeighbors(AtmBuffers A, AtmConfig C) {
    if (*(volatile int*)A.flag == 0) return;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= C.numSites) return;
    const int a = warp;
    const int molA = A.molecule[a];
    int count = 0;
    for (int b0 = a + 1; b0 < C.numSites; b0 += 32) {
        const int b = b0 + lane;
        bool near = false;
        if (b < C.numSites && A.molecule[b] != molA) {
            double d[3];
            siteDelta(A, C, a, b, d);
            near = (float)(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) < C.listCutoff2;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, near);
        if (near) {
            const int k = count + __popc(bal & laneMaskLt());
            if (k < A.cap) A.nbr[(size_t)a * A.cap + k] = b;
        }
        count += __popc(bal);
    }
    if (lane == 0) {
        A.nbrCount[a] = min(count, A.cap);
        if (count > A.cap) atomicOr(A.flag + 1, 1);
    }
    for (int d = 0; d < 3; d++)
        if (lane == 0) A.siteRef[3 * a + d] = A.sitePos[3 * a + d];
}

// Tang-Toennies f_3 and its derivative (InteraxThreeBodyTerms.h:51-65); the series is exact to float for x < 2 at
// k = 16.
__device__ __forceinline__ void tangToennies3f(float x, float& f, float& df) {
    const float e = expNeg(x);
    const float t3 = x * x * x * (1.0f / 6.0f);
    df = e * t3;
    if (x < 2.0f) {
        float term = t3, tail = 0.0f;
#pragma unroll
        for (int k = 4; k <= 16; k++) {
            term *= x * (1.0f / k);
            tail += term;
        }
        f = e * tail;
    }
    else f = fmaf(-e, ((1.0f + x) + 0.5f * x * x) + t3, 1.0f);
}

// g = 1 - exp(-(r/R0)^6) and g' (InteraxThreeBodyTerms.h:71-77).
__device__ __forceinline__ void centroidDampingF(float r, float invR0, float& g, float& dg) {
    const float x = r * invR0;
    float x6 = x * x * x;
    x6 *= x6;
    const float e = expNeg(x6);
    g = x6 < 0.01f ? x6 * fmaf(-0.5f * x6, fmaf(-x6, 1.0f / 3.0f, 1.0f), 1.0f) : 1.0f - e;
    dg = 6.0f * x6 * e * rcpApprox(r);
}

struct AtmWarpStorage {
    float dx[256], dy[256], dz[256];
    float4 params[256];
    int mol[256];
    int site[256];
    float fx[256], fy[256], fz[256];
};

constexpr int kAtmWarps = 4;
constexpr int kAtmMaxStaged = 256;

__global__ void __launch_bounds__(32 * kAtmWarps) kTriples(AtmBuffers A, AtmConfig C) {
    extern __shared__ unsigned char atmShared[];
    AtmWarpStorage& S = reinterpret_cast<AtmWarpStorage*>(atmShared)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    double eAcc = 0.0;
    unsigned long long triples = 0;
    for (int a = blockIdx.x * kAtmWarps + (threadIdx.x >> 5); a < C.numSites; a += gridDim.x * kAtmWarps) {
        const int n = A.nbrCount[a];
        const float4 pa = A.siteParams[a];
        // stage the neighbors within the cutoff
        int m = 0;
        for (int k0 = 0; k0 < n; k0 += 32) {
            const int k = k0 + lane;
            bool in = false;
            double d[3];
            int b = -1;
            if (k < n) {
                b = A.nbr[(size_t)a * A.cap + k];
                siteDelta(A, C, a, b, d);
                in = (float)(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) < C.cutoff2;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, in);
            if (in) {
                const int slot = m + __popc(bal & laneMaskLt());
                if (slot < kAtmMaxStaged) {
                    S.dx[slot] = (float)d[0];
                    S.dy[slot] = (float)d[1];
                    S.dz[slot] = (float)d[2];
                    S.params[slot] = A.siteParams[b];
                    S.mol[slot] = A.molecule[b];
                    S.site[slot] = b;
                    S.fx[slot] = 0.0f;
                    S.fy[slot] = 0.0f;
                    S.fz[slot] = 0.0f;
                }
            }
            m += __popc(bal);
        }
        if (m > kAtmMaxStaged) {
            if (lane == 0) atomicOr(A.flag + 1, 2);
            m = kAtmMaxStaged;
        }
        __syncwarp();
        float fax = 0.0f, fay = 0.0f, faz = 0.0f;
        const int numPairs = m * (m - 1) / 2;
        for (int p = lane; p < numPairs; p += 32) {
            // p = c (c - 1)/2 + b with b < c
            int c = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)p)) * 0.5f);
            while (c * (c - 1) / 2 > p) c--;
            while ((c + 1) * c / 2 <= p) c++;
            const int b = p - c * (c - 1) / 2;
            if (S.mol[b] == S.mol[c]) continue;
            // a = AB, b = AC, c = BC (minimum image of C - B)
            const float ax = S.dx[b], ay = S.dy[b], az = S.dz[b];
            const float bx = S.dx[c], by = S.dy[c], bz = S.dz[c];
            float cx = bx - ax, cy = by - ay, cz = bz - az;
            if (C.periodic) minimumImageF(cx, cy, cz, C.boxf);
            const float w = fmaf(cx, cx, fmaf(cy, cy, cz * cz));
            if (!(w < C.cutoff2)) continue;
            const float4 pb = S.params[b], pc = S.params[c];
            // C9 (InteraxThreeBodyForceImpl.h:69-72), scale and alchemical factor (ReferenceInteraxThreeBodyIxn.cpp:116-120)
            const float wa = pa.y, wb = pb.y, wc = pc.y;
            float c9 = 1.5f * pa.x * pb.x * pc.x * wa * wb * wc * ((wa + wb) + wc) *
                       __fdividef(1.0f, (wa + wb) * (wb + wc) * (wc + wa)) * C.scale;
            if (pa.w != 0.0f || pb.w != 0.0f || pc.w != 0.0f) c9 *= C.lambda;
            if (c9 == 0.0f) continue;
            const float u = fmaf(ax, ax, fmaf(ay, ay, az * az));
            const float v = fmaf(bx, bx, fmaf(by, by, bz * bz));
            const float pp = fmaf(ax, bx, fmaf(ay, by, az * bz));
            const float qq = fmaf(ax, cx, fmaf(ay, cy, az * cz));
            const float ss = fmaf(bx, cx, fmaf(by, cy, bz * cz));
            const float P = u * v * w;
            const float y = rsqrtApprox(P);
            const float invP = y * y;
            const float invP32 = invP * y;
            const float invP52 = invP32 * invP;
            const float pqs = pp * qq * ss;
            float energy = c9 * fmaf(-3.0f * pqs, invP52, invP32);
            const float radial = c9 * fmaf(15.0f * pqs, invP52, -3.0f * invP32);
            const float cross = -3.0f * c9 * invP52;
            const float ru = radial * rcpApprox(u), rv = radial * rcpApprox(v), rw = radial * rcpApprox(w);
            float gax = ax * ru + (bx * (qq * ss) + cx * (pp * ss)) * cross;
            float gay = ay * ru + (by * (qq * ss) + cy * (pp * ss)) * cross;
            float gaz = az * ru + (bz * (qq * ss) + cz * (pp * ss)) * cross;
            float gbx = bx * rv + (ax * (qq * ss) + cx * (pp * qq)) * cross;
            float gby = by * rv + (ay * (qq * ss) + cy * (pp * qq)) * cross;
            float gbz = bz * rv + (az * (qq * ss) + cz * (pp * qq)) * cross;
            float gcx = cx * rw + (ax * (pp * ss) + bx * (pp * qq)) * cross;
            float gcy = cy * rw + (ay * (pp * ss) + by * (pp * qq)) * cross;
            float gcz = cz * rw + (az * (pp * ss) + bz * (pp * qq)) * cross;
            if (C.useTangToennies || C.invCentroidRadius > 0.0f) {
                float len[3], invLen[3];
                len[0] = sqrtRefined(u, invLen[0]);
                len[1] = sqrtRefined(v, invLen[1]);
                len[2] = sqrtRefined(w, invLen[2]);
                const float widths[3] = {pa.z + pb.z, pa.z + pc.z, pb.z + pc.z};
                float f[3], dfdr[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    if (C.useTangToennies) {
                        const float rate = C.twoBeta * __fdividef(1.0f, widths[k]);
                        tangToennies3f(rate * len[k], f[k], dfdr[k]);
                        dfdr[k] *= rate;
                    }
                    else {
                        f[k] = 1.0f;
                        dfdr[k] = 0.0f;
                    }
                    if (C.invCentroidRadius > 0.0f) {
                        float g, dg;
                        centroidDampingF(len[k], C.invCentroidRadius, g, dg);
                        dfdr[k] = fmaf(dfdr[k], g, f[k] * dg);
                        f[k] *= g;
                    }
                }
                const float damping = f[0] * f[1] * f[2];
                const float sa = energy * dfdr[0] * f[1] * f[2] * invLen[0];
                const float sb = energy * f[0] * dfdr[1] * f[2] * invLen[1];
                const float sc = energy * f[0] * f[1] * dfdr[2] * invLen[2];
                gax = fmaf(gax, damping, ax * sa);
                gay = fmaf(gay, damping, ay * sa);
                gaz = fmaf(gaz, damping, az * sa);
                gbx = fmaf(gbx, damping, bx * sb);
                gby = fmaf(gby, damping, by * sb);
                gbz = fmaf(gbz, damping, bz * sb);
                gcx = fmaf(gcx, damping, cx * sc);
                gcy = fmaf(gcy, damping, cy * sc);
                gcz = fmaf(gcz, damping, cz * sc);
                energy *= damping;
            }
            // forceA += dEda + dEdb; forceB += dEdc - dEda; forceC -= dEdb + dEdc (InteraxThreeBodyTerms.h:142-144)
            fax += gax + gbx;
            fay += gay + gby;
            faz += gaz + gbz;
            atomicAdd(&S.fx[b], gcx - gax);
            atomicAdd(&S.fy[b], gcy - gay);
            atomicAdd(&S.fz[b], gcz - gaz);
            atomicAdd(&S.fx[c], -(gbx + gcx));
            atomicAdd(&S.fy[c], -(gby + gcy));
            atomicAdd(&S.fz[c], -(gbz + gcz));
            eAcc += energy;
            triples++;
        }
        __syncwarp();
        for (int k = lane; k < m; k += 32) {
            const int b = S.site[k];
            if (S.fx[k] != 0.0f) atomicAddFixed(A.siteForce + b, toFixed(S.fx[k]));
            if (S.fy[k] != 0.0f) atomicAddFixed(A.siteForce + C.numSites + b, toFixed(S.fy[k]));
            if (S.fz[k] != 0.0f) atomicAddFixed(A.siteForce + 2 * C.numSites + b, toFixed(S.fz[k]));
        }
        for (int o = 16; o > 0; o >>= 1) {
            fax += __shfl_xor_sync(0xffffffffu, fax, o);
            fay += __shfl_xor_sync(0xffffffffu, fay, o);
            faz += __shfl_xor_sync(0xffffffffu, faz, o);
        }
        if (lane == 0) {
            if (fax != 0.0f) atomicAddFixed(A.siteForce + a, toFixed(fax));
            if (fay != 0.0f) atomicAddFixed(A.siteForce + C.numSites + a, toFixed(fay));
            if (faz != 0.0f) atomicAddFixed(A.siteForce + 2 * C.numSites + a, toFixed(faz));
        }
        __syncwarp();
    }
    const double sum = warpSumD(eAcc);
    if (lane == 0) A.energyPartials[blockIdx.x * kAtmWarps + (threadIdx.x >> 5)] = sum;
    for (int o = 16; o > 0; o >>= 1) triples += __shfl_xor_sync(0xffffffffu, triples, o);
    if (lane == 0 && triples) atomicAdd(A.tripleCount, triples);
}

// Each particle of a site receives the site force divided by the number of particles
// (ReferenceInteraxThreeBodyIxn.cpp:127-133).
__global__ void kSpreadSiteForces(AtmBuffers A, AtmConfig C) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C.numSites) return;
    const int b = A.siteOffsets[s], e = A.siteOffsets[s + 1];
    const double inv = 1.0 / (double)(e - b);
    for (int d = 0; d < 3; d++) {
        const long long v = A.siteForce[d * C.numSites + s];
        if (v == 0) continue;
        const long long share = __double2ll_rn((double)v * inv);
        for (int k = b; k < e; k++) atomicAddFixed(A.particleForce + (size_t)d * A.numParticles + A.siteParticles[k], share);
    }
}

}  // namespace ix
