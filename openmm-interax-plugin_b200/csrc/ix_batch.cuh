// Batched evaluation of many independent small systems (clusters, dimer scans, lambda-window copies) in one pass.
// Included at the end of ix_context.cu, whose host helpers it reuses.
//
// The systems' particles are laid out one system after another, each starting on a block of 32 (padding slots fill
// the last block of a system).  The tiles are the block pairs (I, J >= I) of each system, with pair masks that hold
// every pair of the system (j after i, not excluded, gated on); the pair kernel applies the exact cutoff test, so a
// cutoff is honoured while the masks, built once, never need a rebuild.  The three-body neighbor lists hold, for each
// site, the later sites of its system in other molecules; the triple kernel applies the cutoff.  So the whole batch
// is one static launch sequence (positions, block centers, pair kernel, three-body kernels, per-system energies),
// captured once into a CUDA graph and replayed per evaluation.  The pair kernel is the context's persistent kernel
// (warps take tiles from a counter), so small and large systems share the GPU without load-balancing by the host.
//
// Energies per system come from the per-tile and per-site energy slots, which are contiguous per system, summed in a
// fixed order; forces go through the 64-bit fixed-point buffers.  A system's results are therefore identical whether
// it is evaluated alone or in any batch.
#pragma once

namespace {

// Slots to global particles: positions in the build frame (no periodic shift), padding slots at the position of the
// first particle of their block (inside the block's box; they never interact).
__global__ void kBatchPositions(ListBuffers L) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= L.np) return;
    int i = L.sortedAtom[s];
    if (i < 0) i = L.sortedAtom[s & ~31];
    const double x = L.pos[3 * i], y = L.pos[3 * i + 1], z = L.pos[3 * i + 2];
    L.spos[3 * s] = x;
    L.spos[3 * s + 1] = y;
    L.spos[3 * s + 2] = z;
    L.sposf[s] = make_float4((float)x, (float)y, (float)z, 0.0f);
}

// Per-system energies (4 per system: dispersion, exchange, short range, three-body) from the tile slots and the site
// slots of the two triple kernels (wideParts per site of the wide kernel's, 0 when it does not run), in a fixed
// order; one thread per system.  Thread 0 also publishes the interaction
// counts and resets the pair kernel's tile counter.
__global__ void kBatchEnergies(int numSystems, const int* tileStart, const double* tileEnergy, const int* siteStart,
                               const double* siteFast, const double* siteWide, int wideParts, double* out,
                               unsigned long long* counts, int* taskCounter) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) {
        counts[2] = counts[0];
        counts[3] = counts[1];
        counts[0] = 0;
        counts[1] = 0;
        *taskCounter = 0;
    }
    if (s >= numSystems) return;
    double e[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = tileStart[s]; t < tileStart[s + 1]; t++)
        for (int k = 0; k < 3; k++) e[k] += tileEnergy[3 * t + k];
    for (int a = siteStart[s]; a < siteStart[s + 1]; a++) {
        e[3] += siteFast[a];
        for (int w = 0; w < wideParts; w++) e[3] += siteWide[(size_t)a * kAtmWideParts + w];
    }
    for (int k = 0; k < 4; k++) out[4 * s + k] = e[k];
}

// Velocity-Verlet halves for a batch: particles whose system has taken its steps (step >= stopStep) stay put.
__global__ void kBatchVerletFirst(int n, double dt, const double* invMass, const double* force, double* vel,
                                  double* pos, const int* stopStep, const int* step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || *step >= stopStep[i]) return;
    const double h = 0.5 * dt * invMass[i];
    for (int d = 0; d < 3; d++) {
        const double v = vel[3 * i + d] + h * force[3 * i + d];
        vel[3 * i + d] = v;
        pos[3 * i + d] += dt * v;
    }
}

__global__ void kBatchVerletSecond(int n, double dt, const double* invMass, const double* force, double* vel,
                                   const int* stopStep, int* step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && *step < stopStep[i]) {
        const double h = 0.5 * dt * invMass[i];
        for (int d = 0; d < 3; d++) vel[3 * i + d] += h * force[3 * i + d];
    }
}

__global__ void kBatchStepDone(int* step) { *step += 1; }

}  // namespace

struct ix_batch {
    int device = 0;
    DeviceArena* arena = nullptr;        // the owning server's device memory (null: cudaMalloc)
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    std::vector<ix_ctx*> systems;        // host-side descriptions (validation and storage of ix_ctx; no device state)
    std::vector<int> particleStart;      // numSystems + 1, global particle index of each system's first particle
    std::map<std::string, double> parameters;
    std::map<std::string, DeviceBuffer> buffers;
    bool built = false;
    bool dirty = true;                   // parameters changed since the device arrays were built
    // device state
    ListBuffers L{};
    PairBuffers P{};
    AtmBuffers A{};
    PairTermConfig pairC{};
    AtmConfig atmC{};
    unsigned terms = 0;
    bool lean = true, table = false, uniform = false;
    unsigned gatesAll = 0, alchAny = 0;  // bit t: every particle has term t's gate; some particle is alchemical in t
    int pairGrid = 0, numTiles = 0, numSites = 0, numParticles = 0;
    int atmFastBlocks = 0, atmWideBlocks = 0;
    int* tileStart = nullptr;            // numSystems + 1
    int* siteStart = nullptr;            // numSystems + 1
    double* tileEnergy = nullptr;
    double* sitePartials = nullptr;
    double* dPos = nullptr;              // numParticles x 3
    double* dForces = nullptr;           // numParticles x 3
    double* dEnergies = nullptr;         // numSystems x 4
    unsigned long long* dCounts = nullptr;
    long long lastPairs = 0, lastTriples = 0;
    cudaGraphExec_t graph = nullptr;
    const double* graphPositions = nullptr;
    double* graphForces = nullptr;
    double* graphEnergies = nullptr;
    // velocity-Verlet MD of the whole batch: each system runs its own number of steps, after which its particles stay
    // where they are (their forces and energies are still evaluated, unchanged)
    double* dVel = nullptr;              // numParticles x 3
    double* dInvMass = nullptr;          // numParticles
    int* dStopStep = nullptr;            // numParticles: steps of the particle's system
    int* dStep = nullptr;                // steps taken so far (device counter)
    cudaGraphExec_t stepGraph = nullptr;
    double stepDt = 0.0;
    // deferUploads: a build's uploads are held on the host (pendingBytes, one entry per upload) until
    // flushBatchUploads copies them asynchronously on the batch's stream from pinned staging, so that the server's
    // worker does not wait for the copy engine; otherwise each upload is a synchronous copy
    struct PendingUpload {
        void* dst;
        size_t offset, bytes;
    };
    bool deferUploads = false;
    std::vector<char> pendingBytes;
    std::vector<PendingUpload> pending;
};

namespace {

int batchFail(ix_batch* b, int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (b) b->error = buf;
    return code;
}

#define IX_BCUDA(b, call)                                                                                       \
    do {                                                                                                        \
        cudaError_t _e = (call);                                                                                \
        if (_e != cudaSuccess) return batchFail(b, IX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
    } while (0)

template <class T>
int batchAlloc(ix_batch* b, const std::string& name, size_t count, T** out) {
    DeviceBuffer& d = b->buffers[name];
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    if (!d.p || d.bytes < bytes) {
        arenaFree(b->arena, d.p);
        d.p = nullptr;
        d.bytes = 0;
        cudaError_t e = arenaMalloc(b->arena, &d.p, bytes);
        if (e != cudaSuccess && b->arena) {
            d.p = nullptr;
            return batchFail(b, IX_ERR_MEMORY, "device memory budget exhausted: %zu bytes (%s) do not fit", bytes,
                             name.c_str());
        }
        if (e != cudaSuccess)
            return batchFail(b, IX_ERR_CUDA, "cudaMalloc of %zu bytes (%s) failed: %s", bytes, name.c_str(),
                             cudaGetErrorString(e));
        d.bytes = bytes;
    }
    *out = reinterpret_cast<T*>(d.p);
    return IX_OK;
}

// Host bytes to the device: held for flushBatchUploads when the batch defers its uploads, else copied synchronously.
inline int batchCopyIn(ix_batch* b, void* dst, const void* src, size_t bytes) {
    if (!bytes) return IX_OK;
    if (b->deferUploads) {
        const size_t offset = (b->pendingBytes.size() + 15) / 16 * 16;
        b->pendingBytes.resize(offset + bytes);
        std::memcpy(b->pendingBytes.data() + offset, src, bytes);
        b->pending.push_back({dst, offset, bytes});
        return IX_OK;
    }
    IX_BCUDA(b, cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return IX_OK;
}

template <class T>
int batchUpload(ix_batch* b, const std::string& name, const std::vector<T>& v, T** out) {
    IX_TRY(batchAlloc(b, name, v.size(), out));
    return batchCopyIn(b, *out, v.data(), v.size() * sizeof(T));
}

// Issue the held uploads of a build on the batch's stream from `pinned` (pinned host memory of at least
// pendingBytes.size() bytes that stays valid until the stream has run them).
int flushBatchUploads(ix_batch* b, char* pinned) {
    if (!b->pendingBytes.empty()) std::memcpy(pinned, b->pendingBytes.data(), b->pendingBytes.size());
    for (const auto& u : b->pending)
        IX_BCUDA(b, cudaMemcpyAsync(u.dst, pinned + u.offset, u.bytes, cudaMemcpyHostToDevice, b->stream));
    b->pending.clear();
    b->pendingBytes.clear();
    return IX_OK;
}

// A system's effect on the forces forwarded from the ix_add_* functions: the first error message moves to the batch.
int batchForward(ix_batch* b, int system, int rc) {
    if (rc != IX_OK) return batchFail(b, rc, "system %d: %s", system, b->systems[system]->error.c_str());
    b->dirty = true;
    return IX_OK;
}

}  // namespace

namespace {

// Whether a system can join a batch: non-periodic pair and three-body forces.
bool batchable(const ix_ctx* c) {
    return !(c->pairShared && c->method == IX_CUTOFF_PERIODIC) && !(c->atmPresent && c->atmPeriodic);
}

// Whether two systems have the same forces with the same settings (what systems of one batch must share).
bool sameBatchSettings(const ix_ctx* c, const ix_ctx* c0) {
    bool same = c->pairShared == c0->pairShared && c->atmPresent == c0->atmPresent;
    if (same && c0->pairShared) same = c->method == c0->method && c->cutoff == c0->cutoff;
    for (int t = 0; t < 3 && same; t++) {
        const PairTerm &T = c->term[t], &T0 = c0->term[t];
        same = T.present == T0.present;
        if (same && T.present)
            same = T.alchName == T0.alchName && T.useSwitch == T0.useSwitch &&
                   T.switchDistance == T0.switchDistance && T.softcoreRadius == T0.softcoreRadius &&
                   T.overlapMethod == T0.overlapMethod && T.dampingScale == T0.dampingScale;
    }
    if (same && c0->atmPresent)
        same = c->atmCutoff == c0->atmCutoff && c->atmScale == c0->atmScale && c->atmDamping == c0->atmDamping &&
               c->atmDampingScale == c0->atmDampingScale && c->atmCentroidRadius == c0->atmCentroidRadius &&
               c->atmAlchName == c0->atmAlchName;
    return same;
}

// Every system must carry the same forces with the same settings: one launch configuration serves them all.
int checkBatchSystems(ix_batch* b) {
    const ix_ctx* c0 = b->systems[0];
    if (c0->pairShared && c0->method == IX_CUTOFF_PERIODIC)
        return batchFail(b, IX_ERR_INVALID, "batched systems must be non-periodic (NoCutoff or CutoffNonPeriodic)");
    if (c0->atmPresent && c0->atmPeriodic)
        return batchFail(b, IX_ERR_INVALID, "batched systems must be non-periodic (three-body force)");
    for (size_t s = 1; s < b->systems.size(); s++)
        if (!sameBatchSettings(b->systems[s], c0))
            return batchFail(b, IX_ERR_INVALID,
                             "system %zu: every system of a batch must have the same forces with the same settings "
                             "(nonbonded method, cutoffs, switching, soft core, overlap method, damping, alchemical "
                             "parameter); only particle parameters, exclusions and sites may differ",
                             s);
    return IX_OK;
}

}  // namespace

namespace {

// Pair arrays of the batch: slots, parameters, tiles (block pairs of each system) and their pair masks.
int buildBatchPairs(ix_batch* b, const std::vector<int>& blockStart, int nb) {
    const int S = (int)b->systems.size(), np = 32 * nb, n = b->numParticles;
    std::vector<int> sortedAtom(np, -1), slotOf(n);
    std::vector<float4> p0(np, make_float4(0, 0, 0, 0)), p1 = p0, p2 = p0, p3 = p0;
    std::vector<int> flags(np, 0);
    std::vector<std::vector<float4>> q0(S), q1(S), q2(S), q3(S);
    std::vector<std::vector<int>> qf(S);
    std::vector<const ix_ctx*> sys(b->systems.begin(), b->systems.end());
    std::vector<std::vector<int>*> fl(S);
    for (int s = 0; s < S; s++) {
        packPairParams(sys[s], q0[s], q1[s], q2[s], q3[s], qf[s]);
        fl[s] = &qf[s];
    }
    std::vector<PairCoef> table;
    const int T = classTableHost(sys, fl, table);
    for (int s = 0; s < S; s++)
        for (int k = 0; k < sys[s]->n; k++) {
            const int slot = 32 * blockStart[s] + k, g = b->particleStart[s] + k;
            sortedAtom[slot] = g;
            slotOf[g] = slot;
            p0[slot] = q0[s][k];
            p1[slot] = q1[s][k];
            p2[slot] = q2[s][k];
            p3[slot] = q3[s][k];
            flags[slot] = qf[s][k];
        }
    // tiles and masks: every pair of a system, j after i, not excluded, gated on for some term.  The rows start from
    // the real j slots after i (every pair gated on when all of the system's particles carry the same gate bits, the
    // usual case; else each pair is tested), then each exclusion clears its bit, then the columns are the transpose.
    std::vector<int> tileJ, tileI, tileStart(S + 1, 0);
    std::vector<unsigned> masks;
    for (int s = 0; s < S; s++) {
        tileStart[s] = (int)tileI.size();
        const ix_ctx* c = sys[s];
        const int b0 = blockStart[s], b1 = blockStart[s + 1];
        int gates = -1;
        bool uniformGates = true;
        for (int k = 0; k < c->n && uniformGates; k++) {
            const int g = flags[32 * b0 + k] & kFlagGates;
            if (gates < 0) gates = g;
            uniformGates = g == gates && g != 0;
        }
        const size_t first = tileI.size();
        for (int I = b0; I < b1; I++)
            for (int J = I; J < b1; J++) {
                unsigned real = 0;
                for (int k = 0; k < 32; k++) {
                    const bool r = sortedAtom[32 * J + k] >= 0;
                    tileJ.push_back(r ? 32 * J + k : -1);
                    real |= (unsigned)r << k;
                }
                unsigned row[32];
                for (int i = 0; i < 32; i++) {
                    const int si = 32 * I + i;
                    row[i] = 0;
                    if (sortedAtom[si] < 0) continue;
                    unsigned m = real & (J > I ? 0xffffffffu : (i == 31 ? 0u : 0xffffffffu << (i + 1)));
                    if (!uniformGates)
                        for (unsigned q = m; q; q &= q - 1) {
                            const int k = __builtin_ctz(q);
                            if (!(flags[si] & flags[32 * J + k] & kFlagGates)) m &= ~(1u << k);
                        }
                    row[i] = m;
                }
                tileI.push_back(I);
                masks.insert(masks.end(), row, row + 32);
                masks.insert(masks.end(), 32, 0u);
            }
        // the tile of blocks (I, J), J >= I, of this system: tiles are numbered I-major from b0
        const int nbs = b1 - b0;
        auto tileOf = [&](int I, int J) {
            const int i = I - b0;
            return first + (size_t)(i * nbs - i * (i - 1) / 2) + (size_t)(J - I);
        };
        for (const auto& e : c->exclusions) {   // local indices, first < second
            const int si = 32 * b0 + e.first, sj = 32 * b0 + e.second;
            masks[64 * tileOf(si / 32, sj / 32) + (si & 31)] &= ~(1u << (sj & 31));
        }
        for (size_t t = first; t < tileI.size(); t++) {
            unsigned* m = &masks[64 * t];
            for (int i = 0; i < 32; i++)
                for (unsigned q = m[i]; q; q &= q - 1) m[32 + __builtin_ctz(q)] |= 1u << i;
        }
    }
    tileStart[S] = (int)tileI.size();
    b->numTiles = (int)tileI.size();
    b->gatesAll = 7u;
    b->alchAny = 0u;
    for (int k = 0; k < np; k++) {
        if (sortedAtom[k] < 0) continue;
        for (int t = 0; t < 3; t++)
            if (!(flags[k] & (kFlagGateDisp << t))) b->gatesAll &= ~(1u << t);
        b->alchAny |= (unsigned)(flags[k] & 7);
    }
    // the pair kernel takes the tiles largest first (see kTileOrder), here ordered once on the host
    std::vector<int> tileOrder(b->numTiles), tilePairs(b->numTiles, 0);
    for (int t = 0; t < b->numTiles; t++) {
        tileOrder[t] = t;
        for (int i = 0; i < 32; i++) tilePairs[t] += __builtin_popcount(masks[64 * (size_t)t + i]);
    }
    std::stable_sort(tileOrder.begin(), tileOrder.end(), [&](int x, int y) { return tilePairs[x] > tilePairs[y]; });
    ListBuffers& L = b->L;
    L.n = n;
    L.nb = nb;
    L.np = np;
    int one = 1;
    IX_TRY(batchUpload(b, "flag", std::vector<int>{one, 0, 0, 0}, &L.flag));   // block boxes every evaluation
    IX_TRY(batchUpload(b, "sortedAtom", sortedAtom, &L.sortedAtom));
    IX_TRY(batchUpload(b, "slotOf", slotOf, &L.slotOf));
    IX_TRY(batchAlloc(b, "spos", 3 * (size_t)np, &L.spos));
    IX_TRY(batchAlloc(b, "sposf", np, &L.sposf));
    IX_TRY(batchAlloc(b, "bbox", 2 * (size_t)nb, &L.bbox));
    IX_TRY(batchUpload(b, "tileJ", tileJ, &L.tileJ));
    IX_TRY(batchUpload(b, "tileIBlock", tileI, &L.tileIBlock));
    IX_TRY(batchUpload(b, "tileMask", masks, &L.tileMask));
    if (b->numTiles > 0) IX_TRY(batchUpload(b, "tileOrder", tileOrder, &L.tileOrder));
    IX_TRY(batchUpload(b, "numTiles", std::vector<int>{b->numTiles}, &L.numTiles));
    IX_TRY(batchUpload(b, "taskCounter", std::vector<int>{0}, &L.taskCounter));
    IX_TRY(batchUpload(b, "tileStart", tileStart, &b->tileStart));
    L.tileCap = std::max(1, b->numTiles);
    L.pos = b->dPos;
    PairBuffers& P = b->P;
    float4 *d0, *d1, *d2, *d3;
    int* df;
    IX_TRY(batchUpload(b, "p0", p0, &d0));
    IX_TRY(batchUpload(b, "p1", p1, &d1));
    IX_TRY(batchUpload(b, "p2", p2, &d2));
    IX_TRY(batchUpload(b, "p3", p3, &d3));
    IX_TRY(batchUpload(b, "flagsSorted", flags, &df));
    P.p0 = d0;
    P.p1 = d1;
    P.p2 = d2;
    P.p3 = d3;
    P.flags = df;
    L.flags = df;
    IX_TRY(batchUpload(b, "forceFixed", std::vector<long long>(3 * (size_t)np, 0), &P.forceFixed));
    IX_TRY(batchAlloc(b, "tileEnergy", 3 * (size_t)std::max(1, b->numTiles), &b->tileEnergy));
    P.taskEnergy = b->tileEnergy;
    P.pairCount = b->dCounts;
    P.coef = nullptr;
    P.numClasses = 0;
    if (T > 0) {
        PairCoef* dTable;
        IX_TRY(batchUpload(b, "classTable", table, &dTable));
        P.coef = dTable;
        P.numClasses = T;
    }
    return IX_OK;
}

}  // namespace

namespace {

// Three-body arrays of the batch: sites of all systems in order, molecules made distinct across systems, and the
// static neighbor lists (the later sites of the same system in other molecules).
int buildBatchSites(ix_batch* b) {
    const int S = (int)b->systems.size();
    std::vector<int> offsets{0}, particles, molecule, siteStart(S + 1, 0);
    std::vector<float4> params;
    std::vector<int> sysOf;
    long long molBase = 0;
    for (int s = 0; s < S; s++) {
        const ix_ctx* c = b->systems[s];
        siteStart[s] = (int)params.size();
        const int ns = c->atmPresent ? (int)c->siteParams.size() / 3 : 0;
        int maxMol = -1;
        for (int k = 0; k < ns; k++) {
            for (int q = c->siteOffsets[k]; q < c->siteOffsets[k + 1]; q++)
                particles.push_back(b->particleStart[s] + c->siteParticles[q]);
            offsets.push_back((int)particles.size());
            const int site = (int)params.size();
            params.push_back(make_float4((float)c->siteParams[3 * k], (float)c->siteParams[3 * k + 1],
                                         (float)c->siteParams[3 * k + 2], c->siteAlch[k] ? 1.0f : 0.0f));
            molecule.push_back(c->molecule[k] < 0 ? -1 - site : (int)(molBase + c->molecule[k]));
            maxMol = std::max(maxMol, c->molecule[k]);
            sysOf.push_back(s);
        }
        molBase += maxMol + 1;
        if (molBase > INT32_MAX) return batchFail(b, IX_ERR_INVALID, "too many molecules in the batch");
    }
    siteStart[S] = (int)params.size();
    const int ns = (int)params.size();
    b->numSites = ns;
    IX_TRY(batchUpload(b, "siteStart", siteStart, &b->siteStart));
    if (ns == 0) return IX_OK;
    std::vector<int> count(ns, 0);
    int cap = 1;
    for (int a = 0; a < ns; a++) {
        for (int c = a + 1; c < siteStart[sysOf[a] + 1]; c++)
            if (molecule[c] != molecule[a]) count[a]++;
        cap = std::max(cap, count[a]);
    }
    cap = (cap + 31) / 32 * 32;
    std::vector<int> nbr((size_t)ns * cap, 0);
    for (int a = 0; a < ns; a++) {
        int k = 0;
        for (int c = a + 1; c < siteStart[sysOf[a] + 1]; c++)
            if (molecule[c] != molecule[a]) nbr[(size_t)a * cap + k++] = c;
    }
    AtmBuffers& A = b->A;
    int *dOff, *dPart, *dMol;
    float4* dParams;
    IX_TRY(batchUpload(b, "siteOffsets", offsets, &dOff));
    IX_TRY(batchUpload(b, "siteParticles", particles, &dPart));
    IX_TRY(batchUpload(b, "siteMolecule", molecule, &dMol));
    IX_TRY(batchUpload(b, "siteParams", params, &dParams));
    A.siteOffsets = dOff;
    A.siteParticles = dPart;
    A.molecule = dMol;
    A.siteParams = dParams;
    IX_TRY(batchAlloc(b, "sitePos", 3 * (size_t)ns, &A.sitePos));
    IX_TRY(batchUpload(b, "siteRef", std::vector<double>(3 * (size_t)ns, 0.0), &A.siteRef));
    IX_TRY(batchUpload(b, "atmFlag", std::vector<int>{0, 0, 0, 0}, &A.flag));
    IX_TRY(batchUpload(b, "nbrCount", count, &A.nbrCount));
    IX_TRY(batchUpload(b, "nbr", nbr, &A.nbr));
    A.cap = cap;
    IX_TRY(batchUpload(b, "siteForce", std::vector<long long>(3 * (size_t)ns, 0), &A.siteForce));
    IX_TRY(batchUpload(b, "atmParticleForce", std::vector<long long>(3 * (size_t)b->numParticles, 0),
                       &A.particleForce));
    A.numParticles = b->numParticles;
    // one warp per site in the fast kernel and one per (site, part) unit in the wide one, so that each site's energy
    // has its own slots
    b->atmFastBlocks = (ns + kAtmFastWarps - 1) / kAtmFastWarps;
    const int wideBlocks = (int)(((size_t)ns * kAtmWideParts + kAtmWarps - 1) / kAtmWarps);
    b->atmWideBlocks = *std::max_element(count.begin(), count.end()) > kAtmFast ? wideBlocks : 0;
    const size_t slots = (size_t)b->atmFastBlocks * kAtmFastWarps + (size_t)wideBlocks * kAtmWarps;
    IX_TRY(batchUpload(b, "sitePartials", std::vector<double>(slots, 0.0), &b->sitePartials));
    A.energyPartials = b->sitePartials;
    A.tripleCount = b->dCounts + 1;
    return IX_OK;
}

}  // namespace

namespace {

// The launch sequence of one batch evaluation (captured into the batch's graph): positions in b->dPos, forces to
// b->dForces, energies to b->dEnergies.
int enqueueBatch(ix_batch* b) {
    cudaStream_t st = b->stream;
    const ListBuffers& L = b->L;
    const int tpb = 256, S = (int)b->systems.size();
    ListGeometry G{};
    G.periodic = 0;
    kBatchPositions<<<(L.np + tpb - 1) / tpb, tpb, 0, st>>>(L);
    kBlockBounds<<<(L.nb * 32 + tpb - 1) / tpb, tpb, 0, st>>>(L, G);
    if (b->numTiles > 0) {
        const PairTermConfig& C = b->pairC;
        if (b->uniform && b->table) kPairTiles<true, true, true><<<b->pairGrid, 32 * kPairWarps, 0, st>>>(L, b->P, C);
        else if (b->uniform) kPairTiles<true, false, true><<<b->pairGrid, 32 * kPairWarps, 0, st>>>(L, b->P, C);
        else if (b->lean && b->table) kPairTiles<true, true><<<b->pairGrid, 32 * kPairWarps, 0, st>>>(L, b->P, C);
        else if (b->lean) kPairTiles<true, false><<<b->pairGrid, 32 * kPairWarps, 0, st>>>(L, b->P, C);
        else if (b->table) kPairTiles<false, true><<<b->pairGrid, 32 * kPairWarps, 0, st>>>(L, b->P, C);
        else kPairTiles<false, false><<<b->pairGrid, 32 * kPairWarps, 0, st>>>(L, b->P, C);
    }
    if (b->numSites > 0) {
        const AtmBuffers& A = b->A;
        const AtmConfig& C = b->atmC;
        const int gS = (b->numSites + tpb - 1) / tpb;
        kSiteCentroids<<<gS, tpb, 0, st>>>(A, C, b->dPos);
        kTriplesFast<<<b->atmFastBlocks, 32 * kAtmFastWarps, 0, st>>>(A, C);
        if (b->atmWideBlocks > 0)
            kTriplesWide<<<b->atmWideBlocks, 32 * kAtmWarps, sizeof(AtmWarpStorage) * kAtmWarps, st>>>(
                A, C, b->atmFastBlocks * kAtmFastWarps, nullptr);
        kSpreadSiteForces<<<gS, tpb, 0, st>>>(A, C);
    }
    kFinalize<<<(b->numParticles + tpb - 1) / tpb, tpb, 0, st>>>(b->numParticles, L.np, L.slotOf, b->P.forceFixed,
                                                                 b->numSites > 0 ? b->A.particleForce : nullptr,
                                                                 b->dForces, nullptr, 0);
    const double* fast = b->sitePartials;
    const double* wide = b->sitePartials ? b->sitePartials + (size_t)b->atmFastBlocks * kAtmFastWarps : nullptr;
    if (!fast) {
        fast = b->tileEnergy;   // no sites: the site ranges are empty and never read
        wide = b->tileEnergy;
    }
    // the wide kernel's slots hold energies only when it runs (a list longer than the fast kernel's)
    kBatchEnergies<<<(S + tpb - 1) / tpb, tpb, 0, st>>>(S, b->tileStart, b->tileEnergy, b->siteStart, fast, wide,
                                                       b->atmWideBlocks > 0 ? kAtmWideParts : 0, b->dEnergies,
                                                       b->dCounts, L.taskCounter);
    IX_BCUDA(b, cudaGetLastError());
    return IX_OK;
}

}  // namespace

namespace {

int buildBatch(ix_batch* b) {
    const int S = (int)b->systems.size();
    if (S == 0) return batchFail(b, IX_ERR_STATE, "the batch has no systems");
    IX_TRY(checkBatchSystems(b));
    IX_BCUDA(b, cudaSetDevice(b->device));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (b->stepGraph) {
        cudaGraphExecDestroy(b->stepGraph);
        b->stepGraph = nullptr;
    }
    for (ix_ctx* c : b->systems)
        for (auto& kv : b->parameters) c->parameters[kv.first] = kv.second;
    const ix_ctx* c0 = b->systems[0];
    b->numParticles = b->particleStart[S];
    std::vector<int> blockStart(S + 1, 0);
    for (int s = 0; s < S; s++) blockStart[s + 1] = blockStart[s] + (b->systems[s]->n + 31) / 32;
    IX_TRY(batchAlloc(b, "positions", 3 * (size_t)b->numParticles, &b->dPos));
    IX_TRY(batchAlloc(b, "forces", 3 * (size_t)b->numParticles, &b->dForces));
    IX_TRY(batchAlloc(b, "energies", 4 * (size_t)S, &b->dEnergies));
    IX_TRY(batchUpload(b, "counts", std::vector<unsigned long long>{0, 0, 0, 0}, &b->dCounts));
    b->terms = 0;
    for (int t = 0; t < 3; t++)
        if (c0->term[t].present) b->terms |= 1u << t;
    IX_TRY(buildBatchPairs(b, blockStart, blockStart[S]));
    IX_TRY(buildBatchSites(b));
    // one configuration for all systems (they share their settings); the overlap is shared only when it is in every
    // system
    ix_ctx* cfg = b->systems[0];
    b->pairC = pairConfig(cfg, b->terms);
    for (int s = 1; s < S && b->pairC.shareOverlap; s++) b->pairC.shareOverlap = pairConfig(b->systems[s], 0).shareOverlap;
    b->pairC.periodic = 0;
    b->lean = true;
    for (int t = 0; t < 3; t++)
        if ((b->terms >> t) & 1u)
            b->lean = b->lean && b->pairC.softShift[t] == 0.0f && !b->pairC.useSwitch[t] && b->pairC.overlapMethod[t] == 0;
    b->table = b->P.coef != nullptr;
    for (int t = 1; t < 3; t++)
        if ((b->terms >> t) & 1u) b->table = b->table && b->pairC.overlapMethod[t] == 0;
    // every pair of every term evaluated unscaled: the instantiation without per-pair gate and scale tests
    b->uniform = b->lean;
    for (int t = 0; t < 3; t++)
        if ((b->terms >> t) & 1u)
            b->uniform = b->uniform && ((b->gatesAll >> t) & 1u) &&
                         (!((b->alchAny >> t) & 1u) || b->pairC.lambda[t] == 1.0f);
    int perSM = 0;
    if (b->lean && b->table) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kPairTiles<true, true>, 32 * kPairWarps, 0);
    else if (b->lean) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kPairTiles<true, false>, 32 * kPairWarps, 0);
    else if (b->table) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kPairTiles<false, true>, 32 * kPairWarps, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kPairTiles<false, false>, 32 * kPairWarps, 0);
    b->pairGrid = std::max(1, std::min(std::max(1, perSM) * b->numSMs, (b->numTiles + kPairWarps - 1) / kPairWarps));
    if (b->numSites > 0) {
        AtmConfig& C = b->atmC;
        C = AtmConfig{};
        C.numSites = b->numSites;
        C.periodic = 0;
        C.cutoff2 = (float)(c0->atmCutoff * c0->atmCutoff);
        C.listCutoff2 = C.cutoff2;
        C.scale = (float)c0->atmScale;
        bool anyAlch = false;
        for (const ix_ctx* c : b->systems) anyAlch = anyAlch || c->atmAnyAlch;
        C.lambda = (float)lambdaOf(cfg, c0->atmAlchName, anyAlch);
        C.useTangToennies = c0->atmDamping == IX_TANG_TOENNIES;
        C.twoBeta = (float)(2.0 * c0->atmDampingScale);
        C.invCentroidRadius = c0->atmCentroidRadius > 0 ? (float)(1.0 / c0->atmCentroidRadius) : 0.0f;
        C.maxMove2 = INFINITY;
    }
    // capture the evaluation once
    IX_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueueBatch(b);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc != IX_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    IX_BCUDA(b, e);
    const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    IX_BCUDA(b, ie);
    b->built = true;
    b->dirty = false;
    return IX_OK;
}

// MD state of the whole batch: masses (numParticles), velocities (numParticles x 3; null = at rest) and the number of
// steps of each system.  Resets the step counter.
int batchMdSetup(ix_batch* b, const double* masses, const double* velocities, const int* steps) {
    if (!b->built || b->dirty) IX_TRY(buildBatch(b));
    const int n = b->numParticles, S = (int)b->systems.size();
    std::vector<double> inv(n);
    for (int i = 0; i < n; i++) {
        if (!(masses[i] >= 0)) return batchFail(b, IX_ERR_INVALID, "Illegal mass for particle %d", i);
        inv[i] = masses[i] > 0 ? 1.0 / masses[i] : 0.0;
    }
    std::vector<int> stop(n);
    for (int s = 0; s < S; s++) {
        if (steps[s] < 0) return batchFail(b, IX_ERR_INVALID, "system %d: negative number of steps", s);
        for (int i = b->particleStart[s]; i < b->particleStart[s + 1]; i++) stop[i] = steps[s];
    }
    const double* oldVel = b->dVel;
    const double* oldInv = b->dInvMass;
    const int* oldStop = b->dStopStep;
    const int* oldStep = b->dStep;
    IX_TRY(batchUpload(b, "invMass", inv, &b->dInvMass));
    IX_TRY(batchUpload(b, "stopStep", stop, &b->dStopStep));
    IX_TRY(batchUpload(b, "step", std::vector<int>{0}, &b->dStep));
    IX_TRY(batchAlloc(b, "velocities", 3 * (size_t)n, &b->dVel));
    if (velocities) IX_TRY(batchCopyIn(b, b->dVel, velocities, 3 * (size_t)n * sizeof(double)));
    else if (b->deferUploads) IX_BCUDA(b, cudaMemsetAsync(b->dVel, 0, 3 * (size_t)n * sizeof(double), b->stream));
    else IX_BCUDA(b, cudaMemset(b->dVel, 0, 3 * (size_t)n * sizeof(double)));
    if (b->stepGraph && (oldVel != b->dVel || oldInv != b->dInvMass || oldStop != b->dStopStep || oldStep != b->dStep)) {
        cudaGraphExecDestroy(b->stepGraph);
        b->stepGraph = nullptr;
    }
    return IX_OK;
}

// Enqueue one MD step of the batch on its stream: a captured graph of the first half-kick and drift, the evaluation
// at the new positions and the second half-kick (systems past their steps stay put), then the step counter.
int batchMdStep(ix_batch* b, double dt) {
    if (b->stepGraph && b->stepDt != dt) {
        cudaGraphExecDestroy(b->stepGraph);
        b->stepGraph = nullptr;
    }
    if (!b->stepGraph) {
        const int n = b->numParticles, g = (n + 255) / 256;
        IX_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        kBatchVerletFirst<<<g, 256, 0, b->stream>>>(n, dt, b->dInvMass, b->dForces, b->dVel, b->dPos, b->dStopStep,
                                                    b->dStep);
        int rc = enqueueBatch(b);
        kBatchVerletSecond<<<g, 256, 0, b->stream>>>(n, dt, b->dInvMass, b->dForces, b->dVel, b->dStopStep, b->dStep);
        kBatchStepDone<<<1, 1, 0, b->stream>>>(b->dStep);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (rc == IX_OK && e != cudaSuccess) rc = batchFail(b, IX_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
        if (rc == IX_OK) {
            const cudaError_t ie = cudaGraphInstantiate(&b->stepGraph, graph, 0);
            if (ie != cudaSuccess) {
                b->stepGraph = nullptr;
                rc = batchFail(b, IX_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(ie));
            }
        }
        if (graph) cudaGraphDestroy(graph);
        if (rc != IX_OK) return rc;
        b->stepDt = dt;
    }
    IX_BCUDA(b, cudaGraphLaunch(b->stepGraph, b->stream));
    return IX_OK;
}

}  // namespace

extern "C" {

int ix_batch_create(int device, ix_batch** out) {
    if (!out) return fail(nullptr, IX_ERR_INVALID, "ix_batch_create: out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(nullptr, IX_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= count)
        return fail(nullptr, IX_ERR_NO_DEVICE, "CUDA device %d does not exist (%d devices)", device, count);
    cudaSetDevice(device);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    if (prop.major < 10)
        return fail(nullptr, IX_ERR_NO_DEVICE, "device %d (%s, sm_%d%d) is not a Blackwell (sm_100) GPU", device,
                    prop.name, prop.major, prop.minor);
    ix_batch* b = new ix_batch();
    b->device = device;
    b->numSMs = prop.multiProcessorCount;
    b->particleStart.push_back(0);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return fail(nullptr, IX_ERR_CUDA, "cudaStreamCreate failed");
    }
    *out = b;
    return IX_OK;
}

void ix_batch_destroy(ix_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->stepGraph) cudaGraphExecDestroy(b->stepGraph);
    for (auto& kv : b->buffers) arenaFree(b->arena, kv.second.p);
    for (ix_ctx* c : b->systems) delete c;   // host-side descriptions only
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* ix_batch_last_error(const ix_batch* b) { return b ? b->error.c_str() : g_createError.c_str(); }

int ix_batch_add_system(ix_batch* b, int num_particles, int* system) {
    if (!b) return IX_ERR_INVALID;
    if (num_particles <= 0) return batchFail(b, IX_ERR_INVALID, "ix_batch_add_system: the system has no particles");
    if (b->particleStart.back() + (long long)num_particles > (1LL << 30))
        return batchFail(b, IX_ERR_INVALID, "ix_batch_add_system: too many particles in the batch");
    ix_ctx* c = new ix_ctx();
    c->n = num_particles;
    c->device = b->device;
    b->systems.push_back(c);
    b->particleStart.push_back(b->particleStart.back() + num_particles);
    b->dirty = true;
    if (system) *system = (int)b->systems.size() - 1;
    return IX_OK;
}

static int batchSystem(ix_batch* b, int system) {
    if (!b) return IX_ERR_INVALID;
    if (system < 0 || system >= (int)b->systems.size())
        return batchFail(b, IX_ERR_INVALID, "system index %d out of range (%zu systems)", system, b->systems.size());
    return IX_OK;
}

int ix_batch_add_dispersion(ix_batch* b, int system, const ix_pair_settings* settings, const double* params,
                            const uint8_t* alch, double damping_scale, int use_lrc) {
    IX_TRY(batchSystem(b, system));
    return batchForward(b, system, ix_add_dispersion(b->systems[system], settings, params, alch, damping_scale, use_lrc));
}

int ix_batch_add_exchange(ix_batch* b, int system, const ix_pair_settings* settings, const double* params,
                          const uint8_t* alch, int overlap_method) {
    IX_TRY(batchSystem(b, system));
    return batchForward(b, system, ix_add_exchange(b->systems[system], settings, params, alch, overlap_method));
}

int ix_batch_add_short_range(ix_batch* b, int system, const ix_pair_settings* settings, const double* params,
                             const uint8_t* alch, int overlap_method) {
    IX_TRY(batchSystem(b, system));
    return batchForward(b, system, ix_add_short_range(b->systems[system], settings, params, alch, overlap_method));
}

int ix_batch_add_three_body(ix_batch* b, int system, int num_sites, const int32_t* site_offsets,
                            const int32_t* site_particles, const double* site_params, const int32_t* molecule,
                            const uint8_t* alch, double cutoff, double scale_factor, int damping_method,
                            double damping_scale, double centroid_radius, int periodic, const char* alch_name,
                            int force_group) {
    IX_TRY(batchSystem(b, system));
    return batchForward(b, system,
                        ix_add_three_body(b->systems[system], num_sites, site_offsets, site_particles, site_params,
                                          molecule, alch, cutoff, scale_factor, damping_method, damping_scale,
                                          centroid_radius, periodic, alch_name, force_group));
}

int ix_batch_set_parameter(ix_batch* b, const char* name, double value) {
    if (!b || !name) return IX_ERR_INVALID;
    b->parameters[name] = value;
    b->dirty = true;
    return IX_OK;
}

int ix_batch_num_particles(const ix_batch* b, int* num_particles, int* num_systems) {
    if (!b) return IX_ERR_INVALID;
    if (num_particles) *num_particles = b->particleStart.back();
    if (num_systems) *num_systems = (int)b->systems.size();
    return IX_OK;
}

void* ix_batch_get_stream(ix_batch* b) { return b ? (void*)b->stream : nullptr; }

int ix_batch_compute_device(ix_batch* b, const double* d_positions, double* d_forces, double* d_energies) {
    NvtxRange nvtxRange("ix_batch_compute_device");
    if (!b) return IX_ERR_INVALID;
    IX_BCUDA(b, cudaSetDevice(b->device));
    if (!b->built || b->dirty) IX_TRY(buildBatch(b));
    const size_t n3 = 3 * (size_t)b->numParticles;
    if (d_positions && d_positions != b->dPos)
        IX_BCUDA(b, cudaMemcpyAsync(b->dPos, d_positions, n3 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    IX_BCUDA(b, cudaGraphLaunch(b->graph, b->stream));
    if (d_forces)
        IX_BCUDA(b, cudaMemcpyAsync(d_forces, b->dForces, n3 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    if (d_energies)
        IX_BCUDA(b, cudaMemcpyAsync(d_energies, b->dEnergies, 4 * b->systems.size() * sizeof(double),
                                    cudaMemcpyDeviceToDevice, b->stream));
    return IX_OK;
}

int ix_batch_compute(ix_batch* b, const double* positions, double* forces, double* energies) {
    NvtxRange nvtxRange("ix_batch_compute");
    if (!b) return IX_ERR_INVALID;
    if (!positions) return batchFail(b, IX_ERR_INVALID, "ix_batch_compute: positions is NULL");
    const size_t n3 = 3 * (size_t)b->particleStart.back();
    for (size_t i = 0; i < n3; i++)
        if (!std::isfinite(positions[i]))
            return batchFail(b, IX_ERR_INVALID, "Particle coordinate is NaN or infinite (particle %zu)", i / 3);
    IX_BCUDA(b, cudaSetDevice(b->device));
    if (!b->built || b->dirty) IX_TRY(buildBatch(b));
    IX_BCUDA(b, cudaMemcpyAsync(b->dPos, positions, n3 * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    IX_TRY(ix_batch_compute_device(b, nullptr, nullptr, nullptr));
    if (forces) IX_BCUDA(b, cudaMemcpyAsync(forces, b->dForces, n3 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    if (energies)
        IX_BCUDA(b, cudaMemcpyAsync(energies, b->dEnergies, 4 * b->systems.size() * sizeof(double),
                                    cudaMemcpyDeviceToHost, b->stream));
    unsigned long long c[4];
    IX_BCUDA(b, cudaMemcpyAsync(c, b->dCounts, sizeof(c), cudaMemcpyDeviceToHost, b->stream));
    IX_BCUDA(b, cudaStreamSynchronize(b->stream));
    b->lastPairs = (long long)c[2];
    b->lastTriples = (long long)c[3];
    return IX_OK;
}

int ix_batch_md_run(ix_batch* b, const int* steps, double dt, const double* masses, double* positions,
                    double* velocities, double* forces, double* energies) {
    if (!b) return IX_ERR_INVALID;
    if (!steps || !masses || !positions) return batchFail(b, IX_ERR_INVALID, "ix_batch_md_run: null argument");
    if (!(dt > 0)) return batchFail(b, IX_ERR_INVALID, "ix_batch_md_run: the step size must be positive");
    const size_t n3 = 3 * (size_t)b->particleStart.back();
    for (size_t i = 0; i < n3; i++)
        if (!std::isfinite(positions[i]))
            return batchFail(b, IX_ERR_INVALID, "Particle coordinate is NaN or infinite (particle %zu)", i / 3);
    IX_BCUDA(b, cudaSetDevice(b->device));
    if (!b->built || b->dirty) IX_TRY(buildBatch(b));
    IX_TRY(batchMdSetup(b, masses, velocities, steps));
    IX_BCUDA(b, cudaMemcpyAsync(b->dPos, positions, n3 * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    IX_BCUDA(b, cudaGraphLaunch(b->graph, b->stream));   // forces at the starting positions
    int maxSteps = 0;
    for (size_t s = 0; s < b->systems.size(); s++) maxSteps = std::max(maxSteps, steps[s]);
    for (int k = 0; k < maxSteps; k++) IX_TRY(batchMdStep(b, dt));
    IX_BCUDA(b, cudaMemcpyAsync(positions, b->dPos, n3 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    if (velocities)
        IX_BCUDA(b, cudaMemcpyAsync(velocities, b->dVel, n3 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    if (forces) IX_BCUDA(b, cudaMemcpyAsync(forces, b->dForces, n3 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    if (energies)
        IX_BCUDA(b, cudaMemcpyAsync(energies, b->dEnergies, 4 * b->systems.size() * sizeof(double),
                                    cudaMemcpyDeviceToHost, b->stream));
    unsigned long long c[4];
    IX_BCUDA(b, cudaMemcpyAsync(c, b->dCounts, sizeof(c), cudaMemcpyDeviceToHost, b->stream));
    IX_BCUDA(b, cudaStreamSynchronize(b->stream));
    b->lastPairs = (long long)c[2];
    b->lastTriples = (long long)c[3];
    return IX_OK;
}

int ix_batch_get_counts(ix_batch* b, long long* num_pairs, long long* num_triples) {
    if (!b) return IX_ERR_INVALID;
    unsigned long long c[4] = {0, 0, 0, 0};
    if (b->built) {
        IX_BCUDA(b, cudaStreamSynchronize(b->stream));
        IX_BCUDA(b, cudaMemcpy(c, b->dCounts, sizeof(c), cudaMemcpyDeviceToHost));
    }
    if (num_pairs) *num_pairs = (long long)c[2];
    if (num_triples) *num_triples = (long long)c[3];
    return IX_OK;
}

}  // extern "C"
