// Device neighbor list of the fused pair pass: a deterministic cell sort of the particles into blocks of 32, block
// bounding boxes, and per i-block lists of "tiles" (one i-block x 32 candidate j particles within cutoff + skin of the
// i-block's box).  Each tile carries its pair masks: bit j of row i is set when the pair (i, j) can interact before
// the next rebuild (within cutoff + skin at build time, not excluded, j after i, some term gated on), and the
// transposed column masks; the pair kernel visits only those pairs and needs no per-step candidate test.  Every
// kernel of the build reads the rebuild flag and returns at once when it is clear, so the whole pipeline can be
// launched every step (and captured in a CUDA graph) without a host round trip.
//
// The reference gets its list from OpenMM (NonbondedUtilities, called at platforms/common/src/
// CommonInteraxKernels.cpp:209) and, on the Reference platform, a voxel hash (ReferenceInteraxPairIxn.h:86-87).
// Any list containing every pair within the cutoff gives the same interacting set once the kernel applies the exact
// r < cutoff test, which it does.
#pragma once

#include "ix_common.cuh"

namespace ix {

constexpr float kPairSkin = IX_TUNE_PAIR_SKIN;   // nm; rebuild when a particle has moved by more than half of it

// Particle flags in the sorted parameter arrays.
constexpr int kFlagReal = 1 << 3;
constexpr int kFlagGateDisp = 1 << 4;    // alpha != 0
constexpr int kFlagGateExch = 1 << 5;    // exchange width != 0
constexpr int kFlagGateSr = 1 << 6;      // short-range width != 0
constexpr int kFlagGates = kFlagGateDisp | kFlagGateExch | kFlagGateSr;

// Frame shared by the build and evaluation kernels.
struct ListGeometry {
    int periodic;          // CutoffPeriodic
    int useCutoff;         // not NoCutoff
    Box box;
    BoxF boxf;
    float listCutoff;      // cutoff + skin (ignored without cutoff)
    int nc[3];             // cell grid
    float invCell[3];      // cells per unit of fractional coordinate (periodic) or per nm (non-periodic)
};

struct ListBuffers {
    int n, nb, np;
    // rebuild control: flag[0] rebuild, flag[1] tile overflow, flag[2..3] unused
    int* flag;
    // original-order input positions and the positions at the last build
    const double* pos;
    double* refPos;
    float* bboxMinMax;          // non-periodic bounding box of all particles (6 floats, as ordered ints)
    // cell sort
    int* cellKey;               // n
    int* cellCount;             // numCells
    int* cellStart;             // numCells + 1
    int* cellFill;              // numCells
    int* order;                 // n: particles in cell order (within a cell by index after the per-cell sort)
    const int* cellRank;        // dense cell index -> rank along the Hilbert curve
    int numCells;
    // sorted particles
    int* sortedAtom;            // np: original index, -1 for padding
    int* slotOf;                // n
    double* shift;              // np x 3: build frame = position - shift
    double* spos;               // np x 3: current position in the build frame
    float4* sposf;              // np
    float4* bbox;               // nb x 2: center (xyz), half extent (xyz)
    // tiles
    int* blockAtoms;            // nb: candidate j particles of each i-block
    int* blockTiles;            // nb + 1: exclusive scan of the tile counts, then the total
    int* tileJ;                 // tileCap x 32
    int* tileIBlock;            // tileCap
    int* tileBucket;            // tileCap: each tile's candidate pairs / 32 (bits 0..5) and its rank in that bucket
    int* bucketCount;           // 33: tiles per bucket
    int* tileOrder;             // tileCap: the tiles by decreasing candidate count, the pair kernel's schedule (null:
                                // list order), so that the last tiles the warps take are short
    unsigned* tileMask;         // tileCap x 64: row masks (per i lane, bit = j slot), then column masks (per j lane)
    int* numTiles;              // tiles to evaluate (0 after an overflow)
    int* taskCounter;           // next tile of the pair kernel's dynamic schedule (zeroed before each launch)
    int tileCap;
    const int* flags;           // sorted particle flags (the term gates of each particle)
    // exclusions (original indices), CSR with sorted partners and their range
    const int* exclStart;
    const int* exclList;
    const int2* exclRange;
};

__device__ __forceinline__ bool rebuildRequested(const ListBuffers& L) { return *(volatile int*)L.flag != 0; }

// Displacement check: any particle moved more than half the skin since the last build sets the rebuild flag.
__global__ void kCheckDisplacement(ListBuffers L, float maxMove2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    if (i < L.n) {
        double dx = L.pos[3 * i] - L.refPos[3 * i];
        double dy = L.pos[3 * i + 1] - L.refPos[3 * i + 1];
        double dz = L.pos[3 * i + 2] - L.refPos[3 * i + 2];
        moved = (float)(dx * dx + dy * dy + dz * dz) > maxMove2;
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) atomicOr(L.flag, 1);
}

// Float as an order-preserving int, so that min/max reductions can use integer atomics.
__device__ __forceinline__ int floatToOrdered(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float orderedToFloat(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void kResetCells(ListBuffers L) {
    if (!rebuildRequested(L)) return;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < L.numCells; c += gridDim.x * blockDim.x) {
        L.cellCount[c] = 0;
        L.cellFill[c] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x < 6) {
        int* mm = reinterpret_cast<int*>(L.bboxMinMax);
        mm[threadIdx.x] = threadIdx.x < 3 ? floatToOrdered(INFINITY) : floatToOrdered(-INFINITY);
    }
}

// Bounding box of all particles (non-periodic cell grids span it).
__global__ void kParticleBounds(ListBuffers L) {
    if (!rebuildRequested(L)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float v[6];
    for (int k = 0; k < 3; k++) {
        float x = i < L.n ? (float)L.pos[3 * i + k] : INFINITY;
        v[k] = warpMinF(x);
        float y = i < L.n ? (float)L.pos[3 * i + k] : -INFINITY;
        v[3 + k] = warpMaxF(y);
    }
    if ((threadIdx.x & 31) == 0) {
        int* mm = reinterpret_cast<int*>(L.bboxMinMax);
        for (int k = 0; k < 3; k++) {
            atomicMin(mm + k, floatToOrdered(v[k]));
            atomicMax(mm + 3 + k, floatToOrdered(v[3 + k]));
        }
    }
}

// Wrap a position into the reduced periodic cell (c, then b, then a), returning the shift (position - wrapped).
__device__ __forceinline__ void wrapIntoCell(const double p[3], const Box& box, double w[3], double s[3]) {
    w[0] = p[0];
    w[1] = p[1];
    w[2] = p[2];
    double k = floor(w[2] * box.inv[2]);
    w[0] -= k * box.c[0];
    w[1] -= k * box.c[1];
    w[2] -= k * box.c[2];
    k = floor(w[1] * box.inv[1]);
    w[0] -= k * box.b[0];
    w[1] -= k * box.b[1];
    k = floor(w[0] * box.inv[0]);
    w[0] -= k * box.a[0];
    for (int d = 0; d < 3; d++) s[d] = p[d] - w[d];
}

__device__ __forceinline__ int cellOf(const double w[3], const ListGeometry& G, const float* mm) {
    int c[3];
    if (G.periodic) {
        // fractional coordinates of the reduced cell
        double fz = w[2] * G.box.inv[2];
        double fy = (w[1] - fz * G.box.c[1]) * G.box.inv[1];
        double fx = (w[0] - fz * G.box.c[0] - fy * G.box.b[0]) * G.box.inv[0];
        double f[3] = {fx, fy, fz};
        for (int d = 0; d < 3; d++) c[d] = min(max((int)(f[d] * G.nc[d]), 0), G.nc[d] - 1);
    }
    else {
        for (int d = 0; d < 3; d++) {
            float lo = orderedToFloat(__float_as_int(mm[d])), hi = orderedToFloat(__float_as_int(mm[3 + d]));
            float ext = fmaxf(hi - lo, 1e-3f);
            c[d] = min(max((int)(((float)w[d] - lo) / ext * G.nc[d]), 0), G.nc[d] - 1);
        }
    }
    return (c[2] * G.nc[1] + c[1]) * G.nc[0] + c[0];
}

__global__ void kCellKeys(ListBuffers L, ListGeometry G) {
    if (!rebuildRequested(L)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    double p[3] = {L.pos[3 * i], L.pos[3 * i + 1], L.pos[3 * i + 2]};
    double w[3], s[3];
    if (G.periodic) wrapIntoCell(p, G.box, w, s);
    else {
        for (int d = 0; d < 3; d++) w[d] = p[d];
    }
    int key = L.cellRank[cellOf(w, G, L.bboxMinMax)];
    L.cellKey[i] = key;
    atomicAdd(L.cellCount + key, 1);
}

// Exclusive scan of the cell counts in one block of 1024 threads.
__global__ void kScanCells(ListBuffers L) {
    if (!rebuildRequested(L)) return;
    __shared__ int partial[1024];
    const int t = threadIdx.x;
    const int per = (L.numCells + 1023) / 1024;
    const int begin = min(t * per, L.numCells), end = min(begin + per, L.numCells);
    int sum = 0;
    for (int c = begin; c < end; c++) sum += L.cellCount[c];
    partial[t] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        int v = t >= off ? partial[t - off] : 0;
        __syncthreads();
        partial[t] += v;
        __syncthreads();
    }
    int run = partial[t] - sum;
    for (int c = begin; c < end; c++) {
        L.cellStart[c] = run;
        run += L.cellCount[c];
    }
    if (t == 1023) L.cellStart[L.numCells] = partial[1023];
}

__global__ void kScatterCells(ListBuffers L) {
    if (!rebuildRequested(L)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    int key = L.cellKey[i];
    int slot = L.cellStart[key] + atomicAdd(L.cellFill + key, 1);
    L.order[slot] = i;
}

// Within each cell, order the particles by index, so that the sorted order does not depend on atomic timing.
__global__ void kSortWithinCells(ListBuffers L) {
    if (!rebuildRequested(L)) return;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= L.numCells) return;
    int b = L.cellStart[c], e = L.cellStart[c + 1];
    for (int i = b + 1; i < e; i++) {
        int v = L.order[i];
        int j = i - 1;
        while (j >= b && L.order[j] > v) {
            L.order[j + 1] = L.order[j];
            j--;
        }
        L.order[j + 1] = v;
    }
}

// Sorted particle data: original index, image shift that places the particle in the build frame, positions.
__global__ void kSortedAtoms(ListBuffers L, ListGeometry G) {
    if (!rebuildRequested(L)) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= L.np) return;
    if (s < L.n) {
        int i = L.order[s];
        L.sortedAtom[s] = i;
        L.slotOf[i] = s;
        double p[3] = {L.pos[3 * i], L.pos[3 * i + 1], L.pos[3 * i + 2]};
        double w[3], sh[3] = {0, 0, 0};
        if (G.periodic) wrapIntoCell(p, G.box, w, sh);
        for (int d = 0; d < 3; d++) {
            L.shift[3 * s + d] = sh[d];
            L.refPos[3 * i + d] = p[d];
        }
    }
    else {
        L.sortedAtom[s] = -1;
        for (int d = 0; d < 3; d++) L.shift[3 * s + d] = 0.0;
    }
}

// Current positions in the build frame (every step, after a possible rebuild).  Padding slots copy the last real
// particle's position, which keeps the blocks' boxes tight; they never interact.
__global__ void kUpdateSortedPositions(ListBuffers L) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= L.np) return;
    int src = s < L.n ? s : L.n - 1;
    int i = L.sortedAtom[src];
    double x = L.pos[3 * i] - L.shift[3 * src];
    double y = L.pos[3 * i + 1] - L.shift[3 * src + 1];
    double z = L.pos[3 * i + 2] - L.shift[3 * src + 2];
    L.spos[3 * s] = x;
    L.spos[3 * s + 1] = y;
    L.spos[3 * s + 2] = z;
    L.sposf[s] = make_float4((float)x, (float)y, (float)z, 0.0f);
}

// Bounding box of each block (one warp per block), from the build-time positions.
// The center's w is 1 when the block's tiles may place each j particle once, at its minimum image relative to the
// block center, instead of taking the minimum image of every pair: that holds in a rectangular periodic box when
// half of every box length exceeds the block's half extent plus the list cutoff plus the skin (room for the motion
// between rebuilds), since then no interacting pair can need a different image.
__global__ void kBlockBounds(ListBuffers L, ListGeometry G) {
    if (!rebuildRequested(L)) return;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= L.nb) return;
    float4 p = L.sposf[warp * 32 + lane];
    float lo[3] = {warpMinF(p.x), warpMinF(p.y), warpMinF(p.z)};
    float hi[3] = {warpMaxF(p.x), warpMaxF(p.y), warpMaxF(p.z)};
    if (lane == 0) {
        const float half[3] = {0.5f * (hi[0] - lo[0]), 0.5f * (hi[1] - lo[1]), 0.5f * (hi[2] - lo[2])};
        float shift = 0.0f;
        if (G.periodic && !G.box.triclinic) {
            const float len[3] = {(float)G.box.a[0], (float)G.box.b[1], (float)G.box.c[2]};
            bool ok = true;
            for (int d = 0; d < 3; d++) ok = ok && (half[d] + G.listCutoff + kPairSkin < 0.4999f * len[d]);
            shift = ok ? 1.0f : 0.0f;
        }
        L.bbox[2 * warp] = make_float4(0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2]), shift);
        L.bbox[2 * warp + 1] = make_float4(half[0], half[1], half[2], 0.0f);
    }
}

// Squared distance between the boxes of two blocks (rectangular minimum image when periodic); 0 if they overlap.
// Triclinic boxes are not pruned (every block is a candidate); the pair kernel's exact test decides.
__device__ __forceinline__ float boxBoxDist2(float4 ci, float4 ei, float4 cj, float4 ej, const ListGeometry& G) {
    float dx = cj.x - ci.x, dy = cj.y - ci.y, dz = cj.z - ci.z;
    if (G.periodic) {
        if (G.box.triclinic) return 0.0f;
        dx -= G.boxf.a[0] * rintf(dx * G.boxf.inv[0]);
        dy -= G.boxf.b[1] * rintf(dy * G.boxf.inv[1]);
        dz -= G.boxf.c[2] * rintf(dz * G.boxf.inv[2]);
    }
    dx = fmaxf(fabsf(dx) - ei.x - ej.x, 0.0f);
    dy = fmaxf(fabsf(dy) - ei.y - ej.y, 0.0f);
    dz = fmaxf(fabsf(dz) - ei.z - ej.z, 0.0f);
    return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ float pointBoxDist2(float4 p, float4 ci, float4 ei, const ListGeometry& G) {
    return boxBoxDist2(ci, ei, p, make_float4(0, 0, 0, 0), G);
}

__device__ __forceinline__ bool isExcluded(const ListBuffers& L, int oi, int oj) {
    int2 range = L.exclRange[oi];
    if (oj < range.x || oj > range.y) return false;
    int lo = L.exclStart[oi], hi = L.exclStart[oi + 1] - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int v = L.exclList[mid];
        if (v == oj) return true;
        if (v < oj) lo = mid + 1;
        else hi = mid - 1;
    }
    return false;
}

constexpr int kListThreads = 256;                 // one thread block of 8 warps per i-block
constexpr int kListWarps = kListThreads / 32;

// Candidate j particles of one i-block (one thread block per i-block): the particles of the blocks J >= I whose box is
// within the list cutoff of block I's box and whose own position is within it too, in the order (J, slot).  The blocks
// are examined 256 at a time: each thread tests one block's box, the candidate blocks are compacted in block order, and
// the warps take them round robin for the particle tests, so that the search of an i-block whose candidates crowd
// into one index range is not serialised on one warp.  PASS 0 counts the candidates; PASS 1 writes their slots to the
// i-block's tile rows and its tile headers.  Both passes make the same decisions, so the lists do not depend on
// scheduling.
template <int PASS>
__global__ void __launch_bounds__(kListThreads) kListTiles(ListBuffers L, ListGeometry G) {
    if (!rebuildRequested(L)) return;
    __shared__ int candJ[kListThreads];
    __shared__ unsigned keep[kListThreads];
    __shared__ int offset[kListThreads];
    __shared__ int warpTotal[kListWarps];
    const int I = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float4 ci = L.bbox[2 * I], ei = L.bbox[2 * I + 1];
    const float cut2 = G.useCutoff ? G.listCutoff * G.listCutoff : INFINITY;
    int t0 = 0, t1 = 0;
    if (PASS == 1) {
        t0 = L.blockTiles[I];
        t1 = L.blockTiles[I + 1];
        if (t1 > L.tileCap) return;   // overflow: nothing is scheduled, the host grows the buffers and builds again
    }
    const long long base = 32LL * t0, last = 32LL * t1;
    int count = 0;
    for (int Jc = I; Jc < L.nb; Jc += kListThreads) {
        // the candidate blocks of this chunk, in block order
        const int J = Jc + tid;
        const bool cand = J < L.nb && boxBoxDist2(ci, ei, L.bbox[2 * J], L.bbox[2 * J + 1], G) < cut2;
        const unsigned b = __ballot_sync(0xffffffffu, cand);
        if (lane == 0) warpTotal[warp] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < kListWarps; w++) {
            const int c = warpTotal[w];
            before += w < warp ? c : 0;
            total += c;
        }
        if (cand) candJ[before + __popc(b & laneMaskLt())] = J;
        __syncthreads();
        // the particle tests of the candidate blocks
        for (int k = warp; k < total; k += kListWarps) {
            const int j = candJ[k] * 32 + lane;
            bool in = L.sortedAtom[j] >= 0;
            if (in && G.useCutoff) in = pointBoxDist2(L.sposf[j], ci, ei, G) < cut2;
            const unsigned m = __ballot_sync(0xffffffffu, in);
            if (lane == 0) keep[k] = m;
        }
        __syncthreads();
        // offsets of the candidate blocks' particles: exclusive scan over the chunk
        const int v = tid < total ? __popc(keep[tid]) : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) warpTotal[warp] = incl;
        __syncthreads();
        int wBefore = 0, chunkAtoms = 0;
        for (int w = 0; w < kListWarps; w++) {
            const int c = warpTotal[w];
            wBefore += w < warp ? c : 0;
            chunkAtoms += c;
        }
        if (tid < total) offset[tid] = count + wBefore + incl - v;
        __syncthreads();
        if (PASS == 1) {
            for (int k = warp; k < total; k += kListWarps) {
                const unsigned m = keep[k];
                const long long pos = base + offset[k] + __popc(m & laneMaskLt());
                if (((m >> lane) & 1u) && pos < last) L.tileJ[pos] = candJ[k] * 32 + lane;
            }
        }
        count += chunkAtoms;
        __syncthreads();   // the shared arrays are refilled by the next chunk
    }
    if (PASS == 0) {
        if (tid == 0) L.blockAtoms[I] = count;
    }
    else {
        // tile headers: the i-block of each tile, padding (-1) after the last candidate of the last tile
        for (int t = t0 + tid; t < t1; t += kListThreads) L.tileIBlock[t] = I;
        const int rest = count & 31;
        if (t1 > t0 && rest != 0 && tid >= rest && tid < 32) L.tileJ[last - 32 + tid] = -1;
    }
}

// Pair masks of the tiles, one warp per tile over the whole list (the tiles of an i-block vary in number, so a
// per-i-block distribution would wait on the largest); lane = the tile's j lane, the i particles from shared memory.
// A pair's bit is set when j's slot follows i's (each pair once), both are real particles gated on for a common term,
// the pair is not excluded and its build-time distance (minimum image) is within the list cutoff: then no pair outside
// the masks can come within the cutoff before the displacement check requests the next build.  The tests that do not
// depend on the distance are masks formed once per tile; where the i-block allows it (rectangular box, block small
// against the box), j is placed at its image nearest the block's center once, as in the pair kernel, instead of a
// minimum image per pair.  Exclusions are looked up only for the pairs whose i lies in j's exclusion range.  Row
// masks: lane = i slot, bit k = the tile's j lane k; column masks: the transpose.
__global__ void __launch_bounds__(kListThreads) kTileMasks(ListBuffers L, ListGeometry G) {
    if (!rebuildRequested(L)) return;
    __shared__ float4 ipos[kListWarps][32];   // xyz and the original index (as its bits)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // the margin covers the float rounding of the build-time distance
    const float cut2 = G.useCutoff ? G.listCutoff * G.listCutoff * (1.0f + 1e-5f) : INFINITY;
    const int numTiles = *L.numTiles;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < numTiles; t += warps) {
        const int I = L.tileIBlock[t];
        const int si = I * 32 + lane;
        const int oi = L.sortedAtom[si];
        const int fi = L.flags[si];
        float4 p = L.sposf[si];
        p.w = __int_as_float(oi);
        __syncwarp();
        ipos[warp][lane] = p;
        __syncwarp();
        const unsigned iReal = __ballot_sync(0xffffffffu, oi >= 0);
        const unsigned gateD = __ballot_sync(0xffffffffu, (fi & kFlagGateDisp) != 0);
        const unsigned gateE = __ballot_sync(0xffffffffu, (fi & kFlagGateExch) != 0);
        const unsigned gateS = __ballot_sync(0xffffffffu, (fi & kFlagGateSr) != 0);
        const int sj = L.tileJ[32LL * t + lane];
        int oj = -1, fj = 0;
        float4 pj = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int2 jr = make_int2(1, 0);
        if (sj >= 0) {
            oj = L.sortedAtom[sj];
            fj = L.flags[sj];
            pj = L.sposf[sj];
            if (oj >= 0) jr = L.exclRange[oj];
        }
        unsigned column = 0;
        if (oj >= 0) {
            column = iReal & (((fj & kFlagGateDisp) ? gateD : 0u) | ((fj & kFlagGateExch) ? gateE : 0u) |
                              ((fj & kFlagGateSr) ? gateS : 0u));
            const int d = sj - I * 32;   // the i slots of the block below j's
            column &= d >= 32 ? 0xffffffffu : (d <= 0 ? 0u : (1u << d) - 1u);
        }
        if (G.useCutoff && __any_sync(0xffffffffu, column != 0)) {
            bool perPair = G.periodic;
            const float4 c = L.bbox[2 * I];
            if (G.periodic && c.w != 0.0f) {
                pj.x -= G.boxf.a[0] * rintf((pj.x - c.x) * G.boxf.inv[0]);
                pj.y -= G.boxf.b[1] * rintf((pj.y - c.y) * G.boxf.inv[1]);
                pj.z -= G.boxf.c[2] * rintf((pj.z - c.z) * G.boxf.inv[2]);
                perPair = false;
            }
            unsigned in = 0;
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float4 q = ipos[warp][i];
                float dx = pj.x - q.x, dy = pj.y - q.y, dz = pj.z - q.z;
                if (perPair) minimumImageF(dx, dy, dz, G.boxf);
                if (fmaf(dx, dx, fmaf(dy, dy, dz * dz)) < cut2) in |= 1u << i;
            }
            column &= in;
        }
        if (jr.x <= jr.y) {
            for (unsigned m = column; m; m &= m - 1) {
                const int i = __ffs(m) - 1;
                const int o = __float_as_int(ipos[warp][i].w);
                if (o >= jr.x && o <= jr.y && isExcluded(L, oj, o)) column &= ~(1u << i);
            }
        }
        unsigned row = 0;
        for (int i = 0; i < 32; i++) {
            const unsigned bits = __ballot_sync(0xffffffffu, (column >> i) & 1u);
            if (lane == i) row = bits;
        }
        L.tileMask[64LL * t + lane] = row;
        L.tileMask[64LL * t + 32 + lane] = column;
        const unsigned pairs = __reduce_add_sync(0xffffffffu, (unsigned)__popc(column));
        if (lane == 0 && L.tileBucket) {
            const int b = (int)(pairs >> 5);
            L.tileBucket[t] = (int)((unsigned)b | ((unsigned)atomicAdd(L.bucketCount + b, 1) << 6));
        }
    }
}

// The pair kernel's schedule: the tiles by decreasing candidate count (a counting sort over 33 buckets of 32 pairs:
// the mask kernel counted each bucket and gave each tile its rank in it; here each tile goes to its bucket's start plus
// its rank).  The warps take tiles from a shared counter, so the kernel ends when the last tile taken ends; short tiles
// last keep that tail short.  The order within a bucket follows the atomics and varies from build to build, which
// changes no result: forces are summed in fixed point and energies go to each tile's own slot.
__global__ void kTileOrder(ListBuffers L) {
    if (!rebuildRequested(L)) return;
    __shared__ int start[33];
    if (threadIdx.x == 0) {
        int run = 0;
        for (int b = 32; b >= 0; b--) {
            start[b] = run;
            run += L.bucketCount[b];
        }
    }
    __syncthreads();
    const int n = *L.numTiles;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const unsigned v = (unsigned)L.tileBucket[t];
        L.tileOrder[start[v & 63u] + (int)(v >> 6)] = t;
    }
}

// The exclusive scan of the i-blocks' tile counts (one block of 1024 threads).  On overflow no tile is scheduled
// (nothing is written beyond the buffers); the host grows them and evaluates again.
__global__ void kScanTiles(ListBuffers L) {
    if (!rebuildRequested(L)) return;
    __shared__ int partial[1024];
    const int t = threadIdx.x;
    const int per = (L.nb + 1023) / 1024;
    const int begin = min(t * per, L.nb), end = min(begin + per, L.nb);
    int sum = 0;
    for (int c = begin; c < end; c++) {
        const int tiles = (L.blockAtoms[c] + 31) / 32;
        L.blockTiles[c] = tiles;
        sum += tiles;
    }
    partial[t] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = t >= off ? partial[t - off] : 0;
        __syncthreads();
        partial[t] += v;
        __syncthreads();
    }
    int run = partial[t] - sum;
    for (int c = begin; c < end; c++) {
        const int k = L.blockTiles[c];
        L.blockTiles[c] = run;
        run += k;
    }
    if (t < 33 && L.bucketCount) L.bucketCount[t] = 0;   // for the mask kernel's tile counts
    if (t == 1023) {
        const int total = partial[1023];
        L.blockTiles[L.nb] = total;
        *L.numTiles = total > L.tileCap ? 0 : total;
        if (total > L.tileCap) atomicOr(L.flag + 1, 1);
    }
}

}  // namespace ix
