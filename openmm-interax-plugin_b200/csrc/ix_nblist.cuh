// Device neighbor list of the fused pair pass: a deterministic cell sort of the particles into blocks of 32, block
// bounding boxes, and per i-block lists of "tiles" (one i-block x 32 candidate j particles within cutoff + skin of the
// i-block's box).  Every kernel of the build reads the rebuild flag and returns at once when it is clear, so the
// whole pipeline can be launched every step (and captured in a CUDA graph) without a host round trip.
//
// The reference gets its list from OpenMM (NonbondedUtilities, called at platforms/common/src/
// CommonInteraxKernels.cpp:209) and, on the Reference platform, a voxel hash (ReferenceInteraxPairIxn.h:86-87).
// Any list containing every pair within the cutoff gives the same interacting set once the kernel applies the exact
// r < cutoff test, which it does.
#pragma once

#include "ix_common.cuh"

namespace ix {

constexpr int kTaskTiles = 1;        // tiles of one i-block handled by one warp task (small tasks: short tail)
constexpr float kPairSkin = 0.1f;    // nm; rebuild when a particle has moved by more than half of it

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
    // rebuild control: flag[0] rebuild, flag[1] tile overflow, flag[2] exclusion-mask overflow, flag[3] task overflow
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
    const int* cellRank;        // dense cell index -> Morton rank
    int numCells;
    // sorted particles
    int* sortedAtom;            // np: original index, -1 for padding
    int* slotOf;                // n
    double* shift;              // np x 3: build frame = position - shift
    double* spos;               // np x 3: current position in the build frame
    float4* sposf;              // np
    float4* bbox;               // nb x 2: center (xyz), half extent (xyz)
    // tiles
    int* blockTiles;            // nb + 1: tile count, then exclusive scan (offsets)
    int* blockTasks;            // nb + 1
    int* tileJ;                 // tileCap x 32
    int* tileIBlock;            // tileCap
    int* tileExcl;              // tileCap: index of the exclusion masks or -1
    unsigned* exclMasks;        // exclCap x 32
    int* exclCounter;
    int2* tasks;                // taskCap: (first tile, number of tiles)
    int* numTasks;
    int* taskCounter;           // next task of the pair kernel's dynamic schedule (zeroed before each launch)
    int tileCap, exclCap, taskCap;
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
    if (blockIdx.x == 0 && threadIdx.x == 0) *L.exclCounter = 0;
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

// Tile construction for one i-block (one warp).  Pass 0 counts the tiles, pass 1 writes them at the block's offset.
// Candidate j particles: those of blocks J >= I whose box is within the list cutoff of block I's box, and whose own
// position is within it too; the diagonal block's pairs are halved in the pair kernel (j slot > i slot).
template <int PASS>
__global__ void kBuildTiles(ListBuffers L, ListGeometry G) {
    if (!rebuildRequested(L)) return;
    __shared__ int buffer[8][64];
    const int warpInBlock = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int I = blockIdx.x * (blockDim.x >> 5) + warpInBlock;
    if (I >= L.nb) return;
    int* buf = buffer[warpInBlock];
    const float4 ci = L.bbox[2 * I], ei = L.bbox[2 * I + 1];
    const float cut2 = G.useCutoff ? G.listCutoff * G.listCutoff : INFINITY;
    int count = 0, tiles = 0;
    int tileBase = PASS == 1 ? L.blockTiles[I] : 0;
    const int oi = L.sortedAtom[I * 32 + lane];
    auto emit = [&](int valid) {
        // the first `valid` entries of buf form a tile
        if (PASS == 1) {
            int t = tileBase + tiles;
            if (t < L.tileCap) {
                int j = lane < valid ? buf[lane] : -1;
                L.tileJ[32 * t + lane] = j;
                if (lane == 0) L.tileIBlock[t] = I;
                // exclusion mask of this lane's i particle against the tile's j slots
                unsigned mask = 0;
                if (oi >= 0) {
                    for (int k = 0; k < valid; k++) {
                        int oj = L.sortedAtom[buf[k]];
                        if (oj >= 0 && isExcluded(L, oi, oj)) mask |= 1u << k;
                    }
                }
                int excl = -1;
                if (__any_sync(0xffffffffu, mask != 0)) {
                    int e = 0;
                    if (lane == 0) e = atomicAdd(L.exclCounter, 1);
                    e = __shfl_sync(0xffffffffu, e, 0);
                    if (e < L.exclCap) {
                        L.exclMasks[32 * e + lane] = mask;
                        excl = e;
                    }
                    else if (lane == 0) atomicOr(L.flag + 2, 1);
                }
                if (lane == 0) L.tileExcl[t] = excl;
            }
            else if (lane == 0) atomicOr(L.flag + 1, 1);
        }
        tiles++;
    };
    for (int J0 = I; J0 < L.nb; J0 += 32) {
        const int Jl = J0 + lane;
        bool cand = false;
        if (Jl < L.nb) cand = boxBoxDist2(ci, ei, L.bbox[2 * Jl], L.bbox[2 * Jl + 1], G) < cut2;
        unsigned cmask = __ballot_sync(0xffffffffu, cand);
        while (cmask) {
            const int J = J0 + __ffs(cmask) - 1;
            cmask &= cmask - 1;
            const int j = J * 32 + lane;
            bool keep = L.sortedAtom[j] >= 0;
            if (keep && G.useCutoff) keep = pointBoxDist2(L.sposf[j], ci, ei, G) < cut2;
            unsigned kmask = __ballot_sync(0xffffffffu, keep);
            if (keep) buf[count + __popc(kmask & laneMaskLt())] = j;
            count += __popc(kmask);
            __syncwarp();
            if (count >= 32) {
                emit(32);
                __syncwarp();
                int rest = count - 32;
                int v = lane < rest ? buf[32 + lane] : 0;
                __syncwarp();
                if (lane < rest) buf[lane] = v;
                __syncwarp();
                count = rest;
            }
        }
    }
    if (count > 0) emit(count);
    if (PASS == 0 && lane == 0) {
        L.blockTiles[I] = tiles;
        L.blockTasks[I] = (tiles + kTaskTiles - 1) / kTaskTiles;
    }
    if (PASS == 1 && lane == 0) {
        int taskBase = L.blockTasks[I];
        for (int k = 0; k * kTaskTiles < tiles; k++) {
            int task = taskBase + k;
            int first = tileBase + k * kTaskTiles;
            int count = min(kTaskTiles, tiles - k * kTaskTiles);
            if (task < L.taskCap && first + count <= L.tileCap) L.tasks[task] = make_int2(first, count);
            else atomicOr(L.flag + 3, 1);
        }
    }
}

// Exclusive scans of the per-block tile and task counts (one block of 1024 threads).
__global__ void kScanBlocks(ListBuffers L) {
    if (!rebuildRequested(L)) return;
    __shared__ int pa[1024], pb[1024];
    const int t = threadIdx.x;
    const int per = (L.nb + 1023) / 1024;
    const int begin = min(t * per, L.nb), end = min(begin + per, L.nb);
    int sa = 0, sb = 0;
    for (int c = begin; c < end; c++) {
        sa += L.blockTiles[c];
        sb += L.blockTasks[c];
    }
    pa[t] = sa;
    pb[t] = sb;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        int va = t >= off ? pa[t - off] : 0;
        int vb = t >= off ? pb[t - off] : 0;
        __syncthreads();
        pa[t] += va;
        pb[t] += vb;
        __syncthreads();
    }
    int ra = pa[t] - sa, rb = pb[t] - sb;
    for (int c = begin; c < end; c++) {
        int na = L.blockTiles[c], nbk = L.blockTasks[c];
        L.blockTiles[c] = ra;
        L.blockTasks[c] = rb;
        ra += na;
        rb += nbk;
    }
    if (t == 1023) {
        L.blockTiles[L.nb] = pa[1023];
        L.blockTasks[L.nb] = pb[1023];
        const bool overflow = pa[1023] > L.tileCap || pb[1023] > L.taskCap;
        // on overflow no task is scheduled (the pass writes no tile beyond the buffers); the host grows the
        // buffers and evaluates again
        *L.numTasks = overflow ? 0 : pb[1023];
        if (pa[1023] > L.tileCap) atomicOr(L.flag + 1, 1);
        if (pb[1023] > L.taskCap) atomicOr(L.flag + 3, 1);
    }
}

}  // namespace ix
