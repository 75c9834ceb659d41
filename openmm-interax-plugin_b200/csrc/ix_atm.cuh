// Axilrod-Teller-Muto three-body kernels (the reference's five-kernel pipeline is
// platforms/common/src/kernels/interaxThreeBody.cc:11-655 with host code CommonInteraxKernels.cpp:386-646; the FP64
// definition is openmmapi/include/internal/InteraxThreeBodyTerms.h:51-146 and
// platforms/reference/src/ReferenceInteraxThreeBodyIxn.cpp:84-135).
//
//   kSiteCentroids       site positions (unweighted centroids, double) and the site rebuild check
//   kSiteNeighbors       (rebuild only) per site A the sites B > A of other molecules within cutoff + skin
//   kTriplesFast         one warp per site A with at most kAtmFast listed neighbors: the neighbors within the cutoff
//                        are staged in shared memory with their double-precision minimum-image displacements from A
//                        (rounded to float); the pairs (B, C) of them are enumerated by a flat triangular index so
//                        that all lanes are busy, in rounds of kAtmRound pairs; each triple is counted once (A
//                        lowest) and evaluated in float; the forces on B and C of each pair are stored and gathered
//                        per staged neighbor in a fixed order (no atomics)
//   kTriplesWide         the same for the rare sites with longer lists (chunked beyond kAtmMaxStaged within the
//                        cutoff, so any length), with the B and C forces accumulated by shared-memory atomics; a
//                        site whose list overflowed its capacity scans every later site instead, so an overflow
//                        never drops a triple
//   kSpreadSiteForces    the site forces, shared equally among each site's particles, into the particle forces
#pragma once

#include "ix_common.cuh"

namespace ix {

constexpr float kSiteSkin = IX_TUNE_SITE_SKIN;

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
    int zeroSlots, zeroOffset;   // energy slots the fast kernel clears (those of a wide kernel that may not run)
};

// Cell grid of the site-list search in a rectangular periodic box whose edges hold at least three cells as wide as
// the list cutoff: every site within the list cutoff of a site lies in its cell or the 26 around it.
struct SiteCells {
    int nc[3];                   // cells per axis; nc[0] = 0: no grid (the chunk scan is used)
    float cellsPerNm[3];
    int* cellStart;              // numCells + 1
    int* cellSites;              // the sites by cell, each cell's in increasing order
    int* siteCell;               // numSites
    float4* wrapped;             // numSites: each site's position wrapped into the box (float), w its molecule (int
                                 // bits), written by the cell sort for the list search
};
constexpr int kSiteCellMax = 8192;   // cells the one-block sort holds in shared memory
// sites up to this count are scattered and ordered in dynamic shared memory by the one-block sort (160 KB)
constexpr int kSiteSortSharedMax = 40000;

struct AtmBuffers {
    const int* siteOffsets;      // numSites + 1
    const int* siteParticles;
    const float4* siteParams;    // alpha, frequency, width, alchemical (0/1)
    const int* molecule;         // effective molecule (negative input already replaced by -1 - site)
    double* sitePos;             // numSites x 3
    double* siteRef;             // numSites x 3, at the last list build
    float4* chunkBox;            // 2 per chunk of 32 consecutive sites: box center (w = 1: usable) and half extents,
                                 // of the positions wrapped into a rectangular box; null: the list search scans all
    int* flag;                   // [0] rebuild, [1] neighbor overflow, [2] a list longer than kAtmFast
    int* nbrCount;               // numSites
    int* nbr;                    // numSites x cap
    int cap;
    long long* siteForce;        // 3 x numSites, SoA fixed point
    long long* particleForce;    // 3 x numParticles, SoA fixed point (original order)
    int numParticles;
    double* energyPartials;      // one per warp of the fast triple kernel's grid, then one per warp of the wide one
    unsigned long long* tripleCount;
    SiteCells cells;
};

constexpr int kAtmFast = IX_TUNE_ATM_FAST;     // neighbor lists up to this length take the fast triple kernel
constexpr int kAtmRound = IX_TUNE_ATM_ROUND;   // (B, C) pairs evaluated before their forces are gathered
constexpr int kAtmAccum = IX_TUNE_ATM_ACCUM;   // 1: B and C forces as fixed-point shared-memory sums (no rounds)
constexpr int kAtmFastWarps = 4;

// The flat triangular index p = c (c - 1) / 2 + b of the pairs b < c < kAtmFast, decoded: b | c << 8.
struct TrianglePairs {
    unsigned short bc[kAtmFast * (kAtmFast - 1) / 2];
};
constexpr TrianglePairs makeTrianglePairs() {
    TrianglePairs t{};
    int p = 0;
    for (int c = 1; c < kAtmFast; c++)
        for (int b = 0; b < c; b++) t.bc[p++] = (unsigned short)(b | (c << 8));
    return t;
}
__device__ const TrianglePairs kTrianglePairs = makeTrianglePairs();

// A site position as float, wrapped into a rectangular periodic box (unchanged otherwise): the frame of the chunk
// boxes, in which the minimum-image distance between a point and a box bounds that to every point in the box.
__device__ __forceinline__ float3 siteWrapped(const AtmConfig& C, double x, double y, double z) {
    float3 p = make_float3((float)x, (float)y, (float)z);
    if (C.periodic && !C.box.triclinic) {
        p.x -= C.boxf.a[0] * floorf(p.x * C.boxf.inv[0]);
        p.y -= C.boxf.b[1] * floorf(p.y * C.boxf.inv[1]);
        p.z -= C.boxf.c[2] * floorf(p.z * C.boxf.inv[2]);
    }
    return p;
}

// Squared minimum-image distance from a point to a box (0 inside it), both in the wrapped frame.
__device__ __forceinline__ float siteBoxDist2(const AtmConfig& C, float3 p, float4 c, float4 e) {
    float dx = c.x - p.x, dy = c.y - p.y, dz = c.z - p.z;
    if (C.periodic) {
        dx -= C.boxf.a[0] * rintf(dx * C.boxf.inv[0]);
        dy -= C.boxf.b[1] * rintf(dy * C.boxf.inv[1]);
        dz -= C.boxf.c[2] * rintf(dz * C.boxf.inv[2]);
    }
    dx = fmaxf(fabsf(dx) - e.x, 0.0f);
    dy = fmaxf(fabsf(dy) - e.y, 0.0f);
    dz = fmaxf(fabsf(dz) - e.z, 0.0f);
    return dx * dx + dy * dy + dz * dz;
}

__global__ void kSiteCentroids(AtmBuffers A, AtmConfig C, const double* pos) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    float3 w = make_float3(INFINITY, INFINITY, INFINITY), wMax = make_float3(-INFINITY, -INFINITY, -INFINITY);
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
            A.siteForce[d * C.numSites + s] = 0;   // the triple kernels of this evaluation accumulate from zero
        }
        const double dx = c[0] - A.siteRef[3 * s], dy = c[1] - A.siteRef[3 * s + 1], dz = c[2] - A.siteRef[3 * s + 2];
        moved = (float)(dx * dx + dy * dy + dz * dz) > C.maxMove2;
        w = siteWrapped(C, c[0], c[1], c[2]);
        wMax = w;
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) atomicOr(A.flag, 1);
    if (A.chunkBox) {
        // the box of this warp's 32 sites (blocks are whole warps, so a warp is one chunk)
        const float lo[3] = {warpMinF(w.x), warpMinF(w.y), warpMinF(w.z)};
        const float hi[3] = {warpMaxF(wMax.x), warpMaxF(wMax.y), warpMaxF(wMax.z)};
        const int chunk = s >> 5;
        if ((threadIdx.x & 31) == 0 && 32 * chunk < C.numSites) {
            // the margin covers the float rounding of the wrapped positions
            const float m = 1e-4f;
            const bool usable = !(C.periodic && C.box.triclinic);
            A.chunkBox[2 * chunk] = make_float4(0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2]),
                                                usable ? 1.0f : 0.0f);
            A.chunkBox[2 * chunk + 1] = make_float4(0.5f * (hi[0] - lo[0]) + m, 0.5f * (hi[1] - lo[1]) + m,
                                                    0.5f * (hi[2] - lo[2]) + m, 0.0f);
        }
    }
}

__device__ __forceinline__ void siteDelta(const AtmBuffers& A, const AtmConfig& C, int from, int to, double d[3]) {
    d[0] = A.sitePos[3 * to] - A.sitePos[3 * from];
    d[1] = A.sitePos[3 * to + 1] - A.sitePos[3 * from + 1];
    d[2] = A.sitePos[3 * to + 2] - A.sitePos[3 * from + 2];
    if (C.periodic) minimumImage(d[0], d[1], d[2], C.box);
}

// One warp per site A scans the sites above it, 32-site chunk by chunk, skipping the chunks whose box is farther
// than the list cutoff from A (when the centroid kernel wrote the chunk boxes).  The list is in increasing site order.
__global__ void kSiteNeighbors(AtmBuffers A, AtmConfig C) {
    if (*(volatile int*)A.flag == 0) return;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= C.numSites) return;
    const int a = warp;
    const int molA = A.molecule[a];
    const float3 pa = siteWrapped(C, A.sitePos[3 * a], A.sitePos[3 * a + 1], A.sitePos[3 * a + 2]);
    const float skip2 = C.listCutoff2 * (1.0f + 1e-4f);
    int count = 0;
    for (int b0 = (a + 1) & ~31; b0 < C.numSites; b0 += 32) {
        if (A.chunkBox) {
            const float4 c = A.chunkBox[2 * (b0 >> 5)];
            if (c.w != 0.0f && siteBoxDist2(C, pa, c, A.chunkBox[2 * (b0 >> 5) + 1]) >= skip2) continue;
        }
        const int b = b0 + lane;
        bool near = false;
        if (b > a && b < C.numSites && A.molecule[b] != molA) {
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
        // the full count: a site whose list overflowed its capacity is found by the wide triple kernel, which then
        // scans every later site instead of reading the list
        A.nbrCount[a] = count;
        if (count > A.cap) atomicOr(A.flag + 1, 1);
        // flag[2]: some site needs the wide triple kernel (cleared before each build)
        if (count > kAtmFast || count > A.cap) atomicOr(A.flag + 2, 1);
    }
    for (int d = 0; d < 3; d++)
        if (lane == 0) A.siteRef[3 * a + d] = A.sitePos[3 * a + d];
}

// The sites binned into the cell grid (rebuild only), in one block: each site's cell from its wrapped position, the
// cell counts in shared memory, their scan, the scatter, and each cell's sites put in increasing order (so that the
// lists built from the cells come out the same on every run).  With `sharedSites` (at most kSiteSortSharedMax sites,
// the launch giving 4 bytes of dynamic shared memory per site) the scatter goes to shared memory and a warp per cell
// writes each site at its rank among the cell's sites; else each cell is insertion-sorted in place in global memory.
__global__ void __launch_bounds__(1024) kSiteCellSort(AtmBuffers A, AtmConfig C, int sharedSites) {
    if (*(volatile int*)A.flag == 0) return;
    __shared__ int count[kSiteCellMax];
    __shared__ int threadSum[1024];
    extern __shared__ int scattered[];
    const SiteCells& G = A.cells;
    const int numCells = G.nc[0] * G.nc[1] * G.nc[2];
    const int t = threadIdx.x, T = blockDim.x;
    for (int c = t; c < numCells; c += T) count[c] = 0;
    __syncthreads();
    for (int s = t; s < C.numSites; s += T) {
        const float3 p = siteWrapped(C, A.sitePos[3 * s], A.sitePos[3 * s + 1], A.sitePos[3 * s + 2]);
        const int cx = min(max((int)(p.x * G.cellsPerNm[0]), 0), G.nc[0] - 1);
        const int cy = min(max((int)(p.y * G.cellsPerNm[1]), 0), G.nc[1] - 1);
        const int cz = min(max((int)(p.z * G.cellsPerNm[2]), 0), G.nc[2] - 1);
        const int cell = (cz * G.nc[1] + cy) * G.nc[0] + cx;
        G.siteCell[s] = cell;
        G.wrapped[s] = make_float4(p.x, p.y, p.z, __int_as_float(A.molecule[s]));
        atomicAdd(&count[cell], 1);
    }
    __syncthreads();
    // exclusive scan: each thread a contiguous chunk of cells, then the chunk sums
    const int per = (numCells + T - 1) / T;
    const int c0 = min(t * per, numCells), c1 = min(c0 + per, numCells);
    int sum = 0;
    for (int c = c0; c < c1; c++) sum += count[c];
    threadSum[t] = sum;
    __syncthreads();
    for (int o = 1; o < T; o <<= 1) {
        const int v = t >= o ? threadSum[t - o] : 0;
        __syncthreads();
        threadSum[t] += v;
        __syncthreads();
    }
    int run = threadSum[t] - sum;
    for (int c = c0; c < c1; c++) {
        const int n = count[c];
        G.cellStart[c] = run;
        count[c] = run;          // the fill position from here on
        run += n;
    }
    if (t == T - 1) G.cellStart[numCells] = run;
    __syncthreads();
    int* dst = sharedSites ? scattered : G.cellSites;
    for (int s = t; s < C.numSites; s += T) dst[atomicAdd(&count[G.siteCell[s]], 1)] = s;
    __syncthreads();
    if (sharedSites) {
        // the sites are distinct, so each one's rank among its cell's sites is its place
        const int warp = t >> 5, lane = t & 31;
        for (int c = warp; c < numCells; c += T >> 5) {
            const int start = G.cellStart[c], n = G.cellStart[c + 1] - start;
            for (int e = lane; e < n; e += 32) {
                const int x = scattered[start + e];
                int rank = 0;
                for (int f = 0; f < n; f++) rank += scattered[start + f] < x;
                G.cellSites[start + rank] = x;
            }
        }
        return;
    }
    // insertion sort of each cell's sites (a few dozen at most)
    for (int c = t; c < numCells; c += T) {
        int* v = G.cellSites + G.cellStart[c];
        const int n = G.cellStart[c + 1] - G.cellStart[c];
        for (int i = 1; i < n; i++) {
            const int x = v[i];
            int j = i - 1;
            while (j >= 0 && v[j] > x) {
                v[j + 1] = v[j];
                j--;
            }
            v[j + 1] = x;
        }
    }
}

// The list search over the cell grid (rebuild only): one warp per site A takes the sites B > A of other molecules
// within the list cutoff from the 27 cells around A's cell, in cell order.  The 27 cells' sites are taken as one
// sequence (a prefix over the cell sizes), so the lanes stay busy across cell boundaries.  The distance test uses the
// float wrapped positions of the cell sort with a margin of 1e-4 of the squared list cutoff, far above their rounding
// (a few 1e-6): the list may hold a pair at the very edge of the list cutoff that the double-precision distance would
// leave out, never the reverse, and the triple kernels test the cutoff itself in double.  The counts and flags are
// those of kSiteNeighbors.  Launched with 256-thread blocks.
__global__ void __launch_bounds__(256) kSiteNeighborsCells(AtmBuffers A, AtmConfig C) {
    if (*(volatile int*)A.flag == 0) return;
    __shared__ int cellFirst[8][32], cellEnd[8][32];   // per warp: each cell's first site and its end in the sequence
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (warp >= C.numSites) return;
    const int a = warp;
    const SiteCells& G = A.cells;
    const float4 pa = G.wrapped[a];
    const int molA = __float_as_int(pa.w);
    const float cut2 = C.listCutoff2 * (1.0f + 1e-4f);
    const int cell = G.siteCell[a];
    const int cx = cell % G.nc[0], cy = (cell / G.nc[0]) % G.nc[1], cz = cell / (G.nc[0] * G.nc[1]);
    // lane k < 27 takes the cell (dx, dy, dz) = (k % 3, k / 3 % 3, k / 9) - 1, the order of three nested loops
    int first = 0, n = 0;
    if (lane < 27) {
        const int x = (cx + lane % 3 - 1 + G.nc[0]) % G.nc[0], y = (cy + lane / 3 % 3 - 1 + G.nc[1]) % G.nc[1],
                  z = (cz + lane / 9 - 1 + G.nc[2]) % G.nc[2];
        const int c = (z * G.nc[1] + y) * G.nc[0] + x;
        first = G.cellStart[c];
        n = G.cellStart[c + 1] - first;
    }
    int end = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, end, o);
        if (lane >= o) end += v;
    }
    const int total = __shfl_sync(0xffffffffu, end, 31);
    cellFirst[w][lane] = first;
    cellEnd[w][lane] = end;
    __syncwarp();
    int count = 0;
    for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        int b = -1;
        if (k < total) {
            // the cell holding entry k: the first whose end exceeds k (binary search over the 27 ends)
            int lo = 0, hi = 26;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (cellEnd[w][mid] > k) hi = mid;
                else lo = mid + 1;
            }
            const int before = lo ? cellEnd[w][lo - 1] : 0;
            b = G.cellSites[cellFirst[w][lo] + (k - before)];
        }
        bool near = false;
        if (b > a) {
            const float4 pb = G.wrapped[b];
            float dx = pb.x - pa.x, dy = pb.y - pa.y, dz = pb.z - pa.z;
            dx -= C.boxf.a[0] * rintf(dx * C.boxf.inv[0]);
            dy -= C.boxf.b[1] * rintf(dy * C.boxf.inv[1]);
            dz -= C.boxf.c[2] * rintf(dz * C.boxf.inv[2]);
            near = __float_as_int(pb.w) != molA && fmaf(dx, dx, fmaf(dy, dy, dz * dz)) < cut2;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, near);
        if (near) {
            const int slot = count + __popc(bal & laneMaskLt());
            if (slot < A.cap) A.nbr[(size_t)a * A.cap + slot] = b;
        }
        count += __popc(bal);
    }
    if (lane == 0) {
        A.nbrCount[a] = count;
        if (count > A.cap) atomicOr(A.flag + 1, 1);
        if (count > kAtmFast || count > A.cap) atomicOr(A.flag + 2, 1);
        for (int d = 0; d < 3; d++) A.siteRef[3 * a + d] = A.sitePos[3 * a + d];
    }
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

// One triple (A, B, C) from the displacements AB = (ax, ay, az) and AC = (bx, by, bz) (minimum images) and the three
// sites' parameters: the C9 coefficient (InteraxThreeBodyForceImpl.h:69-72) with the scale and alchemical factor
// (ReferenceInteraxThreeBodyIxn.cpp:116-120), the ATM energy and its gradients (InteraxThreeBodyTerms.h:97-146),
// optionally Tang-Toennies and centroid damping.  Returns false when BC is outside the cutoff or C9 vanishes.
// fA, fB, fC: the forces on the three sites.
__device__ __forceinline__ bool atmTriple(const AtmConfig& C, const float4& pa, const float4& pb, const float4& pc,
                                          float ax, float ay, float az, float bx, float by, float bz, float& energy,
                                          float3& fA, float3& fB, float3& fC) {
    // a = AB, b = AC, c = BC (minimum image of C - B)
    float cx = bx - ax, cy = by - ay, cz = bz - az;
    if (C.periodic) minimumImageF(cx, cy, cz, C.boxf);
    const float w = fmaf(cx, cx, fmaf(cy, cy, cz * cz));
    if (!(w < C.cutoff2)) return false;
    const float wa = pa.y, wb = pb.y, wc = pc.y;
    float c9 = 1.5f * pa.x * pb.x * pc.x * wa * wb * wc * ((wa + wb) + wc) *
               __fdividef(1.0f, (wa + wb) * (wb + wc) * (wc + wa)) * C.scale;
    if (pa.w != 0.0f || pb.w != 0.0f || pc.w != 0.0f) c9 *= C.lambda;
    if (c9 == 0.0f) return false;
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
    energy = c9 * fmaf(-3.0f * pqs, invP52, invP32);
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
    fA = make_float3(gax + gbx, gay + gby, gaz + gbz);
    fB = make_float3(gcx - gax, gcy - gay, gcz - gaz);
    fC = make_float3(-(gbx + gcx), -(gby + gcy), -(gbz + gcz));
    return true;
}

// Stage the neighbors of site a that are within the cutoff (in list order) with their displacements from a and their
// parameters; returns how many there are (at most `capacity` are stored).
template <class Store>
__device__ __forceinline__ int stageTripleNeighbors(const AtmBuffers& A, const AtmConfig& C, int a, int n, int lane,
                                                    int first, int capacity, Store store) {
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
            const int slot = m + __popc(bal & laneMaskLt()) - first;
            if (slot >= 0 && slot < capacity) store(slot, b, (float)d[0], (float)d[1], (float)d[2]);
        }
        m += __popc(bal);
    }
    return m;
}

// The same for a site whose list overflowed its capacity: every later site of another molecule is tested against the
// cutoff, which gives the same neighbors within the cutoff (in increasing order), so the same triples are evaluated.
// The reference falls back the same way
// (platforms/common/src/kernels/interaxThreeBody.cc:111-112, 437-438).
template <class Store>
__device__ __forceinline__ int stageTripleNeighborsScan(const AtmBuffers& A, const AtmConfig& C, int a, int lane,
                                                        int first, int capacity, Store store) {
    const int molA = A.molecule[a];
    int m = 0;
    for (int b0 = a + 1; b0 < C.numSites; b0 += 32) {
        const int b = b0 + lane;
        bool in = false;
        double d[3];
        if (b < C.numSites && A.molecule[b] != molA) {
            siteDelta(A, C, a, b, d);
            in = (float)(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) < C.cutoff2;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (in) {
            const int slot = m + __popc(bal & laneMaskLt()) - first;
            if (slot >= 0 && slot < capacity) store(slot, b, (float)d[0], (float)d[1], (float)d[2]);
        }
        m += __popc(bal);
    }
    return m;
}

struct AtmFastStorage {
    float4 pos[kAtmFast];        // displacement from A; w holds the molecule (int bits)
    float4 params[kAtmFast];
    int site[kAtmFast];
    float4 fb[kAtmAccum ? 1 : kAtmRound];   // force on B of each pair of the current round
    float4 fc[kAtmAccum ? 1 : kAtmRound];   // force on C
    unsigned long long acc[kAtmAccum ? 3 : 1][kAtmAccum ? kAtmFast : 1];   // fixed-point force sums per neighbor
};

__global__ void __launch_bounds__(32 * kAtmFastWarps, IX_TUNE_ATM_MIN_BLOCKS) kTriplesFast(AtmBuffers A, AtmConfig C) {
    __shared__ AtmFastStorage storage[kAtmFastWarps];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C.zeroSlots; k += gridDim.x * blockDim.x)
        A.energyPartials[C.zeroOffset + k] = 0.0;
    AtmFastStorage& S = storage[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * kAtmFastWarps + (threadIdx.x >> 5);
    double eAcc = 0.0;
    unsigned long long triples = 0;
    for (int a = warp; a < C.numSites; a += gridDim.x * kAtmFastWarps) {
        const int n = A.nbrCount[a];
        if (n > kAtmFast || n > A.cap) continue;      // the wide kernel takes this site
        const float4 pa = A.siteParams[a];
        __syncwarp();
        const int m = stageTripleNeighbors(A, C, a, n, lane, 0, kAtmFast,
                                           [&](int slot, int b, float x, float y, float z) {
                                               S.pos[slot] = make_float4(x, y, z, __int_as_float(A.molecule[b]));
                                               S.params[slot] = A.siteParams[b];
                                               S.site[slot] = b;
                                           });
        __syncwarp();
        float fa[3] = {0.0f, 0.0f, 0.0f};
        float f0[3] = {0.0f, 0.0f, 0.0f}, f1[3] = {0.0f, 0.0f, 0.0f};   // staged neighbors lane, lane + 32
        float eSite = 0.0f;
        int next0 = lane + 1, next1 = lane + 33;    // next C of the pairs (k, C) each lane gathers as B
        const int numPairs = m * (m - 1) / 2;
        if constexpr (kAtmAccum) {
            // each triple's B and C forces go to the neighbors' fixed-point sums (integer adds: the order of the
            // lanes does not change them), flushed once per site
            for (int k = lane; k < m; k += 32) S.acc[0][k] = S.acc[1][k] = S.acc[2][k] = 0ull;
            __syncwarp();
            for (int q = lane; q < numPairs; q += 32) {
                const unsigned bc = __ldg(kTrianglePairs.bc + q);
                const int b = bc & 0xff, c = bc >> 8;
                const float4 xb = S.pos[b], xc = S.pos[c];
                if (__float_as_int(xb.w) == __float_as_int(xc.w)) continue;
                float e;
                float3 fA, fB, fC;
                if (!atmTriple(C, pa, S.params[b], S.params[c], xb.x, xb.y, xb.z, xc.x, xc.y, xc.z, e, fA, fB, fC))
                    continue;
                fa[0] += fA.x;
                fa[1] += fA.y;
                fa[2] += fA.z;
                eSite += e;
                triples++;
                atomicAdd(&S.acc[0][b], (unsigned long long)toFixed(fB.x));
                atomicAdd(&S.acc[1][b], (unsigned long long)toFixed(fB.y));
                atomicAdd(&S.acc[2][b], (unsigned long long)toFixed(fB.z));
                atomicAdd(&S.acc[0][c], (unsigned long long)toFixed(fC.x));
                atomicAdd(&S.acc[1][c], (unsigned long long)toFixed(fC.y));
                atomicAdd(&S.acc[2][c], (unsigned long long)toFixed(fC.z));
            }
            __syncwarp();
            for (int k = lane; k < m; k += 32) {
                const int b = S.site[k];
                for (int d = 0; d < 3; d++)
                    if (S.acc[d][k]) atomicAddFixed(A.siteForce + d * C.numSites + b, (long long)S.acc[d][k]);
            }
        }
        else
        for (int base = 0; base < numPairs; base += kAtmRound) {
            const int count = min(kAtmRound, numPairs - base);
            for (int q = lane; q < count; q += 32) {
                const unsigned bc = __ldg(kTrianglePairs.bc + base + q);
                const int b = bc & 0xff, c = bc >> 8;
                const float4 xb = S.pos[b], xc = S.pos[c];
                float3 fB = make_float3(0.0f, 0.0f, 0.0f), fC = fB;
                if (__float_as_int(xb.w) != __float_as_int(xc.w)) {
                    float e;
                    float3 fA;
                    if (atmTriple(C, pa, S.params[b], S.params[c], xb.x, xb.y, xb.z, xc.x, xc.y, xc.z, e, fA, fB, fC)) {
                        fa[0] += fA.x;
                        fa[1] += fA.y;
                        fa[2] += fA.z;
                        eSite += e;
                        triples++;
                    }
                    else fB = fC = make_float3(0.0f, 0.0f, 0.0f);
                }
                S.fb[q] = make_float4(fB.x, fB.y, fB.z, 0.0f);
                S.fc[q] = make_float4(fC.x, fC.y, fC.z, 0.0f);
            }
            __syncwarp();
            // gather, for the staged neighbors k = lane and lane + 32: the pairs (b, k) with b < k (contiguous) and
            // the pairs (k, c) with c > k (increasing p as c grows)
            auto gather = [&](int k, float f[3], int& next) {
                if (k >= m) return;
                const int first = k * (k - 1) / 2;
                const int lo = max(first, base), hi = min(first + k, base + count);
                for (int p = lo; p < hi; p++) {
                    const float4 v = S.fc[p - base];
                    f[0] += v.x;
                    f[1] += v.y;
                    f[2] += v.z;
                }
                for (; next < m; next++) {
                    const int p = next * (next - 1) / 2 + k;
                    if (p >= base + count) break;
                    const float4 v = S.fb[p - base];
                    f[0] += v.x;
                    f[1] += v.y;
                    f[2] += v.z;
                }
            };
            gather(lane, f0, next0);
            gather(lane + 32, f1, next1);
            __syncwarp();
        }
        // the staged neighbors' forces, then A's (a fixed reduction tree over the lanes)
        auto flush = [&](int k, const float f[3]) {
            if (k >= m) return;
            const int b = S.site[k];
            if (f[0] != 0.0f) atomicAddFixed(A.siteForce + b, toFixed(f[0]));
            if (f[1] != 0.0f) atomicAddFixed(A.siteForce + C.numSites + b, toFixed(f[1]));
            if (f[2] != 0.0f) atomicAddFixed(A.siteForce + 2 * C.numSites + b, toFixed(f[2]));
        };
        if constexpr (!kAtmAccum) {
            flush(lane, f0);
            flush(lane + 32, f1);
        }
        for (int o = 16; o > 0; o >>= 1) {
            fa[0] += __shfl_xor_sync(0xffffffffu, fa[0], o);
            fa[1] += __shfl_xor_sync(0xffffffffu, fa[1], o);
            fa[2] += __shfl_xor_sync(0xffffffffu, fa[2], o);
        }
        if (lane == 0) {
            if (fa[0] != 0.0f) atomicAddFixed(A.siteForce + a, toFixed(fa[0]));
            if (fa[1] != 0.0f) atomicAddFixed(A.siteForce + C.numSites + a, toFixed(fa[1]));
            if (fa[2] != 0.0f) atomicAddFixed(A.siteForce + 2 * C.numSites + a, toFixed(fa[2]));
        }
        eAcc += (double)eSite;
    }
    const double sum = warpSumD(eAcc);
    if (lane == 0) A.energyPartials[warp] = sum;
    for (int o = 16; o > 0; o >>= 1) triples += __shfl_xor_sync(0xffffffffu, triples, o);
    if (lane == 0 && triples) atomicAdd(A.tripleCount, triples);
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
constexpr int kAtmChunk = kAtmMaxStaged / 2;
// Each long-list site is taken by this many warps, each evaluating every kAtmWideParts-th group of 32 of its pairs:
// a site near the start of a large cluster has tens of thousands of (B, C) pairs, which one warp would take alone.
constexpr int kAtmWideParts = 8;

// Sites whose lists are longer than kAtmFast, in units (site, part) of kAtmWideParts parts per site.  A unit stages up
// to kAtmMaxStaged neighbors within the cutoff at once and evaluates its part of their pairs, enumerated by a flat
// triangular index; a longer list is taken in chunks of kAtmChunk, each pair of chunks (I <= J) staged side by side,
// so any length is handled.  The forces on B and C accumulate in shared memory and are flushed to the fixed-point
// site forces after each staging (integer sums: the split changes no result's dependence on the order).  Energies go
// to energyPartials[partialsOffset + warp]: with a grid of one warp per unit, one slot per unit (unit = site x
// kAtmWideParts + part).
// `gate` (may be null): the kernel returns at once unless *gate is set (a list longer than kAtmFast exists).
__global__ void __launch_bounds__(32 * kAtmWarps) kTriplesWide(AtmBuffers A, AtmConfig C, int partialsOffset,
                                                               const int* gate) {
    if (gate && *(volatile const int*)gate == 0) return;
    extern __shared__ unsigned char atmShared[];
    AtmWarpStorage& S = reinterpret_cast<AtmWarpStorage*>(atmShared)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    double eAcc = 0.0;
    unsigned long long triples = 0;
    const int units = C.numSites * kAtmWideParts;
    for (int u = blockIdx.x * kAtmWarps + (threadIdx.x >> 5); u < units; u += gridDim.x * kAtmWarps) {
        const int a = u / kAtmWideParts, part = u % kAtmWideParts;
        const int n = A.nbrCount[a];
        if (n <= kAtmFast && n <= A.cap) continue;     // the fast kernel takes this site
        const float4 pa = A.siteParams[a];
        const bool scan = n > A.cap;                   // the list overflowed: scan every later site
        auto stage = [&](int first, int base, int capacity) {
            auto store = [&](int slot, int b, float x, float y, float z) {
                const int k = base + slot;
                S.dx[k] = x;
                S.dy[k] = y;
                S.dz[k] = z;
                S.params[k] = A.siteParams[b];
                S.mol[k] = A.molecule[b];
                S.site[k] = b;
                S.fx[k] = 0.0f;
                S.fy[k] = 0.0f;
                S.fz[k] = 0.0f;
            };
            return scan ? stageTripleNeighborsScan(A, C, a, lane, first, capacity, store)
                        : stageTripleNeighbors(A, C, a, n, lane, first, capacity, store);
        };
        float fax = 0.0f, fay = 0.0f, faz = 0.0f;
        auto pair = [&](int b, int c) {
            if (S.mol[b] == S.mol[c]) return;
            float energy;
            float3 fA, fB, fC;
            if (!atmTriple(C, pa, S.params[b], S.params[c], S.dx[b], S.dy[b], S.dz[b], S.dx[c], S.dy[c], S.dz[c],
                           energy, fA, fB, fC))
                return;
            fax += fA.x;
            fay += fA.y;
            faz += fA.z;
            atomicAdd(&S.fx[b], fB.x);
            atomicAdd(&S.fy[b], fB.y);
            atomicAdd(&S.fz[b], fB.z);
            atomicAdd(&S.fx[c], fC.x);
            atomicAdd(&S.fy[c], fC.y);
            atomicAdd(&S.fz[c], fC.z);
            eAcc += energy;
            triples++;
        };
        auto triangle = [&](int m) {
            const int numPairs = m * (m - 1) / 2;
            for (int p = lane + 32 * part; p < numPairs; p += 32 * kAtmWideParts) {
                // p = c (c - 1)/2 + b with b < c
                int c = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)p)) * 0.5f);
                while (c * (c - 1) / 2 > p) c--;
                while ((c + 1) * c / 2 <= p) c++;
                pair(p - c * (c - 1) / 2, c);
            }
        };
        auto flush = [&](int lo, int hi) {
            for (int k = lo + lane; k < hi; k += 32) {
                const int b = S.site[k];
                if (S.fx[k] != 0.0f) atomicAddFixed(A.siteForce + b, toFixed(S.fx[k]));
                if (S.fy[k] != 0.0f) atomicAddFixed(A.siteForce + C.numSites + b, toFixed(S.fy[k]));
                if (S.fz[k] != 0.0f) atomicAddFixed(A.siteForce + 2 * C.numSites + b, toFixed(S.fz[k]));
            }
        };
        __syncwarp();
        const int m = stage(0, 0, kAtmMaxStaged);
        __syncwarp();
        if (m <= kAtmMaxStaged) {
            triangle(m);
            __syncwarp();
            flush(0, m);
        }
        else {
            const int chunks = (m + kAtmChunk - 1) / kAtmChunk;
            for (int I = 0; I < chunks; I++) {
                const int cI = min(kAtmChunk, m - I * kAtmChunk);
                for (int J = I; J < chunks; J++) {
                    const int cJ = min(kAtmChunk, m - J * kAtmChunk);
                    __syncwarp();
                    stage(I * kAtmChunk, 0, kAtmChunk);
                    if (J != I) stage(J * kAtmChunk, kAtmChunk, kAtmChunk);
                    __syncwarp();
                    if (J == I) triangle(cI);
                    else
                        for (int p = lane + 32 * part; p < cI * cJ; p += 32 * kAtmWideParts)
                            pair(p / cJ, kAtmChunk + p % cJ);
                    __syncwarp();
                    flush(0, cI);
                    if (J != I) flush(kAtmChunk, kAtmChunk + cJ);
                }
            }
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
    if (lane == 0) A.energyPartials[partialsOffset + blockIdx.x * kAtmWarps + (threadIdx.x >> 5)] = sum;
    for (int o = 16; o > 0; o >>= 1) triples += __shfl_xor_sync(0xffffffffu, triples, o);
    if (lane == 0 && triples) atomicAdd(A.tripleCount, triples);
}

// Each particle of a site receives the site force divided by the number of particles
// (ReferenceInteraxThreeBodyIxn.cpp:127-133).  The site forces are cleared as they are read.
__global__ void kSpreadSiteForces(AtmBuffers A, AtmConfig C) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= C.numSites) return;
    const int b = A.siteOffsets[s], e = A.siteOffsets[s + 1];
    const double inv = 1.0 / (double)(e - b);
    for (int d = 0; d < 3; d++) {
        const long long v = A.siteForce[d * C.numSites + s];
        if (v == 0) continue;
        A.siteForce[d * C.numSites + s] = 0;
        const long long share = __double2ll_rn((double)v * inv);
        for (int k = b; k < e; k++) atomicAddFixed(A.particleForce + (size_t)d * A.numParticles + A.siteParticles[k], share);
    }
}

}  // namespace ix
