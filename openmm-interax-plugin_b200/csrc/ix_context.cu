// Context and C ABI of the B200 kernels (include/interax_b200.h).
//
// A context holds one System's short-range forces on one GPU: the settings and parameters of the three pair forces
// (evaluated together by the fused pair kernel) and of the three-body force, the device buffers, and the CUDA stream
// every launch goes to.  The host logic mirrors the reference's ForceImpl/kernel classes: validation as
// checkPairForce (openmmapi/src/InteraxPairForce.cpp:113-136) and InteraxThreeBodyForceImpl::initialize
// (openmmapi/src/InteraxThreeBodyForceImpl.cpp:42-62), force-group gating as calcForcesAndEnergy
// (InteraxPairForceImpl.h:84-88), parameter updates as copyParametersToContext (ReferenceInteraxKernels.cpp:98-198).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/interax_b200.h"
#include "ix_atm.cuh"
#include "ix_common.cuh"
#include "ix_host_math.h"
#include "ix_md.cuh"
#include "ix_nblist.cuh"
#include "ix_pair.cuh"
#include "ix_probe.cuh"

using namespace ix;

namespace {

thread_local std::string g_createError;

const char* kTermNames[3] = {"InteraxDispersionForce", "InteraxExchangeForce", "InteraxShortRangeForce"};

struct PairTerm {
    bool present = false;
    int group = 0;
    std::string alchName = "lambda_sterics";
    bool useSwitch = false;
    double switchDistance = -1.0, softcoreRadius = 0.0;
    std::vector<double> params;          // n x stride
    std::vector<unsigned char> alch;
    bool anyAlch = false;
    int overlapMethod = 0;
    double dampingScale = 1.0;
    bool useLrc = false;
    double lrcCoef = 0.0, lrcAlchCoef = 0.0;
};

struct DeviceBuffer {
    void* p = nullptr;
    size_t bytes = 0;
};

// Free ranges of memory chunks, best fit by size (O(log n) per allocation and release, however fragmented), with
// neighbouring free ranges of the same chunk merged on release.
struct RangeHeap {
    struct Range {
        size_t bytes;
        int chunk;
    };
    std::map<char*, Range> byAddr;                 // free ranges
    std::multimap<size_t, char*> bySize;           // the same, by size
    std::map<char*, Range> live;                   // allocations

    void addFree(char* p, size_t bytes, int chunk) {
        byAddr[p] = {bytes, chunk};
        bySize.emplace(bytes, p);
    }
    void eraseFree(std::map<char*, Range>::iterator it) {
        auto range = bySize.equal_range(it->second.bytes);
        for (auto s = range.first; s != range.second; ++s)
            if (s->second == it->first) {
                bySize.erase(s);
                break;
            }
        byAddr.erase(it);
    }
    char* take(size_t bytes) {
        auto s = bySize.lower_bound(bytes);
        if (s == bySize.end()) return nullptr;
        char* p = s->second;
        auto it = byAddr.find(p);
        const Range r = it->second;
        eraseFree(it);
        if (r.bytes > bytes) addFree(p + bytes, r.bytes - bytes, r.chunk);
        live[p] = {bytes, r.chunk};
        return p;
    }
    size_t give(char* p) {   // returns the bytes released (0: not an allocation of this heap)
        auto it = live.find(p);
        if (it == live.end()) return 0;
        Range r = it->second;
        const size_t released = r.bytes;
        live.erase(it);
        auto next = byAddr.find(p + r.bytes);
        if (next != byAddr.end() && next->second.chunk == r.chunk) {
            r.bytes += next->second.bytes;
            eraseFree(next);
        }
        auto after = byAddr.lower_bound(p);
        if (after != byAddr.begin()) {
            auto prev = std::prev(after);
            if (prev->second.chunk == r.chunk && prev->first + prev->second.bytes == p) {
                char* q = prev->first;
                const size_t merged = prev->second.bytes + r.bytes;
                eraseFree(prev);
                addFree(q, merged, r.chunk);
                return released;
            }
        }
        addFree(p, r.bytes, r.chunk);
        return released;
    }
};

// Device memory of the contexts and batches a server runs.  Chunks come from cudaMalloc and are sub-allocated on
// the host; they go back to the driver only when the arena is destroyed, because cudaFree waits for the whole device
// and would stall every request in flight.  Live bytes are bounded by the budget (`limit`).
struct DeviceArena {
    static constexpr size_t kAlign = 512;
    std::mutex m;
    std::vector<char*> chunks;
    RangeHeap heap;
    size_t limit = 0, chunkBytes = size_t(256) << 20, inUse = 0, peak = 0, capacity = 0;

    // Add a chunk of `bytes` (cudaMalloc of a large chunk waits for the device, so a server adds its first chunk
    // before it runs anything).
    bool grow(size_t bytes) {
        char* base = nullptr;
        if (cudaMalloc(reinterpret_cast<void**>(&base), bytes) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        chunks.push_back(base);
        capacity += bytes;
        heap.addFree(base, bytes, (int)chunks.size() - 1);
        return true;
    }

    void* alloc(size_t bytes) {
        bytes = (std::max<size_t>(bytes, 1) + kAlign - 1) / kAlign * kAlign;
        std::lock_guard<std::mutex> lock(m);
        if (inUse + bytes > limit) return nullptr;
        char* p = heap.take(bytes);
        if (!p) {
            const size_t want = std::max(chunkBytes, bytes);
            if (capacity + want > limit + chunkBytes || !grow(want)) return nullptr;
            p = heap.take(bytes);
        }
        inUse += bytes;
        peak = std::max(peak, inUse);
        return p;
    }

    void release(void* ptr) {
        std::lock_guard<std::mutex> lock(m);
        inUse -= heap.give(static_cast<char*>(ptr));
    }

    ~DeviceArena() {
        for (char* c : chunks) cudaFree(c);
    }
};

// Device allocation through an arena when one is given, else straight from the driver.
inline cudaError_t arenaMalloc(DeviceArena* arena, void** p, size_t bytes) {
    if (!arena) return cudaMalloc(p, bytes);
    *p = arena->alloc(bytes);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}

inline void arenaFree(DeviceArena* arena, void* p) {
    if (!p) return;
    if (arena) arena->release(p);
    else cudaFree(p);
}

// What a captured graph was captured for: the selected terms, the output pointers and the MD time step.
struct GraphKey {
    unsigned terms = 0;
    const void* out0 = nullptr;
    const void* out1 = nullptr;
    const void* out2 = nullptr;
    const void* out3 = nullptr;
    const void* in0 = nullptr;           // device inputs read by a captured gather (positions in a caller's layout)
    const void* in1 = nullptr;
    const void* in2 = nullptr;
    int format = 0;
    int stride = 0;
    double dt = 0.0;
    double param = 0.0;                  // value of the window parameter a window graph was captured with
    bool operator==(const GraphKey& o) const {
        return terms == o.terms && out0 == o.out0 && out1 == o.out1 && out2 == o.out2 && out3 == o.out3 &&
               in0 == o.in0 && in1 == o.in1 && in2 == o.in2 && format == o.format && stride == o.stride &&
               dt == o.dt && std::memcmp(&param, &o.param, sizeof(param)) == 0;
    }
};

struct LaunchGraph {
    cudaGraphExec_t exec = nullptr;
    GraphKey key;
    unsigned long long version = 0;
    long long launches = 0;              // kernels in the graph
};

}  // namespace

struct ix_ctx {
    int n = 0;
    int device = 0;
    DeviceArena* arena = nullptr;        // the owning server's device memory (null: cudaMalloc)
    std::vector<double> requestPos, requestVel, requestMass;   // starting state of a server request description
    char* uploadBuf = nullptr;           // pinned host staging of a server's context (null: pageable copies)
    unsigned char* hostStatus = nullptr; // pinned host copy of the status block (flags, energies, counts)
    size_t uploadCap = 0, uploadUsed = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;      // the three-body chain, forked from and joined back into `stream`
    cudaStream_t streamBody = nullptr;   // captures the branches of conditional graph nodes
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    bool capturing = false;              // launches are being captured into a graph
    int numSMs = 148;
    std::string error;
    double defaultBox[9] = {2, 0, 0, 0, 2, 0, 0, 0, 2};
    double box[9] = {2, 0, 0, 0, 2, 0, 0, 0, 2};
    bool havePositions = false;
    std::map<std::string, double> parameters;
    bool counting = false;
    long long lastPairs = 0, lastTriples = 0;

    // pair forces
    PairTerm term[3];
    bool pairShared = false;             // method, cutoff and exclusions recorded
    int method = 0;
    double cutoff = 1.0;
    std::vector<std::pair<int, int>> exclusions;   // normalized (min, max), sorted unique
    bool pairDirty = true;               // parameters must be re-uploaded
    unsigned pairGatesAll = 0;           // bit t: every particle takes part in pair term t
    unsigned pairAlchAny = 0;            // bit t: some particle is alchemical in pair term t
    mutable int pairShareOverlap = -1;   // exchange and short-range widths agree for every particle (-1: not known)
    bool pairAllocated = false;
    long long tileCapRequest = 0;        // ix_set_list_capacity: tile capacity of the next allocation (0: estimated)

    // three-body force
    bool atmPresent = false;
    int atmGroup = 0;
    std::string atmAlchName = "lambda_sterics";
    std::vector<int> siteOffsets, siteParticles, molecule;
    std::vector<double> siteParams;      // numSites x 3
    std::vector<unsigned char> siteAlch;
    bool atmAnyAlch = false;
    double atmCutoff = 1.2, atmScale = 1.0, atmDampingScale = 1.0, atmCentroidRadius = 0.0;
    int atmDamping = 0;
    bool atmPeriodic = false;
    bool atmDirty = true;
    bool atmAllocated = false;
    int atmCap = 0;

    // device memory
    std::map<std::string, DeviceBuffer> buffers;
    double* dPos = nullptr;              // n x 3
    unsigned long long* dCounts = nullptr;   // pairs, triples being counted; then those of the last evaluation
    int* dFlags = nullptr;               // pair list flags [4], atm flags [2]
    double* dOutForces = nullptr;        // n x 3
    double* dOutEnergy = nullptr;        // 4
    double* dEnergyBlocks = nullptr;     // kReduceBlocks x 4 partial sums of the energy reduction
    unsigned* dReduceTicket = nullptr;   // blocks of the energy reduction done (the last one finishes, then resets)
    // pair list
    ListBuffers L{};
    ListGeometry G{};
    PairBuffers P{};
    float4 *dP0o = nullptr, *dP1o = nullptr, *dP2o = nullptr, *dP3o = nullptr;
    float4* dP3 = nullptr;
    double* dPairPartials = nullptr;     // per-warp energies of the pair kernel (3 per warp)
    double* dAtmPartials = nullptr;      // per-warp energies of the triple kernel
    int* dParticleSiteStart = nullptr;   // n + 1: the sites of each particle (CSR)
    int* dParticleSites = nullptr;
    int atmFastBlocks = 0;               // grid of the fast triple kernel
    int atmGridBlocks = 0;               // grid of the wide triple kernel
    int* dFlagso = nullptr;
    float4 *dP0 = nullptr, *dP1 = nullptr, *dP2 = nullptr;
    int* dFlagsSorted = nullptr;
    int tileCap = 0;
    int pairGridBlocks = 0;              // persistent grid of the general pair kernel
    int pairGridBlocksLean = 0;          // and of its lean instantiation
    // three-body
    AtmBuffers A{};
    // MD
    double* dVel = nullptr;
    double* dInvMass = nullptr;
    bool haveMasses = false;
    bool mdForcesValid = false;          // dOutForces holds all-group forces of the current positions
    // the state before the enqueued steps not yet finished (positions, velocities, forces: 3n each; energies: 4), so
    // that steps run with an overflowed pair list are rerun from it after the list has grown
    double* dMdSave = nullptr;
    bool mdRollback = true;              // a server's contexts rerun a whole request instead
    long long mdReruns = 0;              // steps rerun after an overflow (ix_get_list_stats)
    bool mdSavedForcesValid = false;
    std::vector<std::pair<int, double>> mdPending;   // steps and dt of each ix_md_steps_async since the save
    // device entry points: the flags of the last call, copied to pinned memory, and the event after the copy
    unsigned char* deviceStatus = nullptr;
    cudaEvent_t evStatus = nullptr;
    bool statusPending = false;
    int lastDeviceStatus = 0;
    int* dAddSlot = nullptr;             // slot in the caller's force buffer of each particle (ix_compute_device_posq)
    // distance constraints of the MD loop (ix_md_set_constraints), as clusters solved by one thread each
    int numConstraints = 0;
    ConstraintClusters K{};
    // optional CUDA-event timing of the pair and triple kernels (ix_set_profiling)
    bool profiling = false;
    bool serialize = false;              // profiling level 2: the three-body chain runs after the pair chain
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool evPair = false, evAtm = false;
    long long launches = 0;              // kernels of this library launched on the context
    // CUDA graphs of the evaluation (host and device entry points) and of one MD step, replayed until a change of
    // state that a captured launch depends on (parameters, box, buffers, settings) bumps the version
    bool useGraphs = true;
    unsigned long long version = 1;
    LaunchGraph graphCompute, graphDevice, graphMd, graphPosq;
    std::vector<LaunchGraph> graphWindows;  // evaluations at window values of one parameter, one graph per value
    size_t windowNext = 0;                  // slot replaced next when graphWindows is full
};

static void bumpVersion(ix_ctx* ctx) {
    if (ctx) ctx->version++;
}

// Energy slots of the triple kernels: one per warp of the fast grid, then one per warp of the wide grid.
static size_t atmPartialCount(const ix_ctx* ctx) {
    return (size_t)ctx->atmFastBlocks * kAtmFastWarps + (size_t)ctx->atmGridBlocks * kAtmWarps;
}

// ---------------------------------------------------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------------------------------------------------

static int fail(ix_ctx* ctx, int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->error = buf;
    else g_createError = buf;
    return code;
}

#define IX_CUDA(ctx, call)                                                                                   \
    do {                                                                                                     \
        cudaError_t _e = (call);                                                                             \
        if (_e != cudaSuccess) return fail(ctx, IX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
    } while (0)

template <class T>
static int deviceAlloc(ix_ctx* ctx, const std::string& name, size_t count, T** out) {
    DeviceBuffer& b = ctx->buffers[name];
    size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    if (b.p && b.bytes >= bytes) {
        *out = reinterpret_cast<T*>(b.p);
        return IX_OK;
    }
    bumpVersion(ctx);
    arenaFree(ctx->arena, b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = arenaMalloc(ctx->arena, &b.p, bytes);
    if (e != cudaSuccess) {
        b.p = nullptr;
        if (ctx->arena)
            return fail(ctx, IX_ERR_MEMORY, "device memory budget exhausted: %zu bytes (%s) do not fit", bytes,
                        name.c_str());
        return fail(ctx, IX_ERR_CUDA, "cudaMalloc of %zu bytes (%s) failed: %s", bytes, name.c_str(),
                    cudaGetErrorString(e));
    }
    b.bytes = bytes;
    *out = reinterpret_cast<T*>(b.p);
    return IX_OK;
}

#define IX_TRY(expr)                \
    do {                            \
        int _rc = (expr);           \
        if (_rc != IX_OK) return _rc; \
    } while (0)

// Copy host data to the device in the context's stream order.  A server's context has pinned staging: the data is
// copied there first and the transfer is asynchronous, with no wait for the stream (a pageable copy waits for the
// stream's earlier work, which on a busy GPU means waiting for other requests' kernels).
static int stageCopy(ix_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (!bytes) return IX_OK;
    if (ctx->uploadBuf && ctx->uploadUsed + bytes <= ctx->uploadCap) {
        char* p = ctx->uploadBuf + ctx->uploadUsed;
        ctx->uploadUsed += (bytes + 63) / 64 * 64;
        std::memcpy(p, src, bytes);
        src = p;
    }
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, IX_ERR_CUDA, "cudaMemcpyAsync failed: %s", cudaGetErrorString(e));
    return IX_OK;
}

// Wait for the uploads just issued (pageable ones only; staged ones stay valid until the stream has run them).
static int uploadsDone(ix_ctx* ctx) {
    if (ctx->uploadBuf) return IX_OK;
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail(ctx, IX_ERR_CUDA, "cudaStreamSynchronize failed: %s", cudaGetErrorString(e));
    return IX_OK;
}


static Box makeBox(const double* b) {
    Box box;
    for (int k = 0; k < 3; k++) {
        box.a[k] = b[k];
        box.b[k] = b[3 + k];
        box.c[k] = b[6 + k];
    }
    box.inv[0] = 1.0 / b[0];
    box.inv[1] = 1.0 / b[4];
    box.inv[2] = 1.0 / b[8];
    box.triclinic = (b[3] != 0 || b[6] != 0 || b[7] != 0);
    return box;
}

static BoxF makeBoxF(const Box& b) {
    BoxF f;
    for (int k = 0; k < 3; k++) {
        f.a[k] = (float)b.a[k];
        f.b[k] = (float)b.b[k];
        f.c[k] = (float)b.c[k];
        f.inv[k] = (float)b.inv[k];
    }
    return f;
}

static double lambdaOf(const ix_ctx* ctx, const std::string& name, bool anyAlch) {
    if (!anyAlch) return 1.0;
    auto it = ctx->parameters.find(name);
    return it == ctx->parameters.end() ? 1.0 : it->second;
}

// Position of cell (x, y, z) on the Hilbert curve through the 2^bits cube (the transpose algorithm of J. Skilling,
// "Programming the Hilbert curve", AIP Conf. Proc. 707, 381 (2004)).  Consecutive cells of the curve are face
// neighbours, so the 32-particle blocks cut from the particles in cell order are compact; a Z-order curve jumps at
// its octant boundaries, and the blocks that straddle a jump span much of the box.
static unsigned long long hilbertIndex(unsigned x, unsigned y, unsigned z, int bits) {
    unsigned X[3] = {x, y, z};
    const unsigned top = 1u << (bits - 1);
    for (unsigned q = top; q > 1; q >>= 1) {
        const unsigned p = q - 1;
        for (int i = 0; i < 3; i++) {
            if (X[i] & q) X[0] ^= p;
            else {
                const unsigned t = (X[0] ^ X[i]) & p;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    for (int i = 1; i < 3; i++) X[i] ^= X[i - 1];
    unsigned t = 0;
    for (unsigned q = top; q > 1; q >>= 1)
        if (X[2] & q) t ^= q - 1;
    for (int i = 0; i < 3; i++) X[i] ^= t;
    unsigned long long h = 0;
    for (int b = bits - 1; b >= 0; b--)
        for (int i = 0; i < 3; i++) h = (h << 1) | ((X[i] >> b) & 1u);
    return h;
}

// The power of two nearest to v (in ratio), within [1, 1024].
static int nearestPow2(double v) {
    int p = 1;
    while (p < 1024 && v >= p * std::sqrt(2.0)) p *= 2;
    return p;
}

// ---------------------------------------------------------------------------------------------------------------------
// pair force setup
// ---------------------------------------------------------------------------------------------------------------------

static int addPairForce(ix_ctx* ctx, int t, const ix_pair_settings* s, const double* params, const uint8_t* alch,
                        int stride) {
    const char* name = kTermNames[t];
    if (!ctx) return IX_ERR_INVALID;
    if (!s || !params || !alch) return fail(ctx, IX_ERR_INVALID, "%s: null argument", name);
    if (ctx->term[t].present) return fail(ctx, IX_ERR_INVALID, "%s: the context already has this force", name);
    // checkPairForce (InteraxPairForce.cpp:113-136)
    if (s->nonbonded_method < 0 || s->nonbonded_method > 2)
        return fail(ctx, IX_ERR_INVALID, "InteraxPairForce: Illegal value for nonbonded method");
    for (int i = 0; i < s->num_exclusions; i++) {
        int p1 = s->exclusions[2 * i], p2 = s->exclusions[2 * i + 1];
        if (p1 < 0 || p1 >= ctx->n || p2 < 0 || p2 >= ctx->n)
            return fail(ctx, IX_ERR_INVALID, "%s: Illegal particle index for an exclusion", name);
    }
    if (s->softcore_radius < 0)
        return fail(ctx, IX_ERR_INVALID, "InteraxPairForce: The soft-core radius cannot be negative");
    if (s->force_group < 0 || s->force_group > 31)
        return fail(ctx, IX_ERR_INVALID, "%s: Force group must be between 0 and 31", name);
    if (s->nonbonded_method != IX_NO_CUTOFF) {
        if (s->cutoff <= 0) return fail(ctx, IX_ERR_INVALID, "%s: The cutoff distance must be positive", name);
        if (s->use_switching_function && (s->switching_distance < 0 || s->switching_distance >= s->cutoff))
            return fail(ctx, IX_ERR_INVALID, "%s: Switching distance must satisfy 0 <= r_switch < r_cutoff", name);
        if (s->nonbonded_method == IX_CUTOFF_PERIODIC) {
            const double* b = ctx->defaultBox;
            if (s->cutoff > 0.5 * b[0] || s->cutoff > 0.5 * b[4] || s->cutoff > 0.5 * b[8])
                return fail(ctx, IX_ERR_INVALID,
                            "%s: The cutoff distance cannot be greater than half the periodic box size.", name);
        }
    }
    // exclusions, normalized
    std::vector<std::pair<int, int>> ex;
    ex.reserve(s->num_exclusions);
    for (int i = 0; i < s->num_exclusions; i++) {
        int p1 = s->exclusions[2 * i], p2 = s->exclusions[2 * i + 1];
        if (p1 != p2) ex.push_back({std::min(p1, p2), std::max(p1, p2)});
    }
    std::sort(ex.begin(), ex.end());
    ex.erase(std::unique(ex.begin(), ex.end()), ex.end());
    double cutoff = s->nonbonded_method == IX_NO_CUTOFF ? 0.0 : s->cutoff;
    if (ctx->pairShared) {
        // one fused pass over one list, as the reference's CUDA platform requires (InteraxPairForce.h:50-53)
        if (ctx->method != s->nonbonded_method || ctx->cutoff != cutoff || ctx->exclusions != ex)
            return fail(ctx, IX_ERR_INVALID,
                        "%s: all Interax pair forces of a Context must have identical nonbonded methods, cutoffs and "
                        "exclusions (they are evaluated in one pass over one neighbor list)",
                        name);
    }
    else {
        ctx->pairShared = true;
        ctx->method = s->nonbonded_method;
        ctx->cutoff = cutoff;
        ctx->exclusions = std::move(ex);
    }
    PairTerm& T = ctx->term[t];
    T.present = true;
    T.group = s->force_group;
    T.alchName = s->alchemical_parameter ? s->alchemical_parameter : "lambda_sterics";
    T.useSwitch = s->nonbonded_method != IX_NO_CUTOFF && s->use_switching_function;
    T.switchDistance = s->switching_distance;
    T.softcoreRadius = s->softcore_radius;
    T.params.assign(params, params + (size_t)ctx->n * stride);
    T.alch.assign(alch, alch + ctx->n);
    T.anyAlch = std::any_of(T.alch.begin(), T.alch.end(), [](unsigned char a) { return a != 0; });
    ctx->pairDirty = true;
    ctx->pairShareOverlap = -1;
    bumpVersion(ctx);
    ctx->pairAllocated = false;
    return IX_OK;
}

static void computeLrc(ix_ctx* ctx) {
    PairTerm& T = ctx->term[0];
    T.lrcCoef = T.lrcAlchCoef = 0.0;
    if (!T.present || !T.useLrc || ctx->method != IX_CUTOFF_PERIODIC) return;
    ixhost::longRangeCorrection(ctx->n, T.params.data(), T.alch.data(), ctx->cutoff, T.useSwitch, T.switchDistance,
                                T.dampingScale, T.lrcCoef, T.lrcAlchCoef);
}

// Per-particle float parameters in original order, with the term flags.
// Coefficients of one ordered pair of overlap widths (w1, w2 > 0), double precision, rounded once to float.
static void overlapCoefficients(double w1, double w2, float4& A, float4& B, float& k1, float& k2, float4& Q,
                                float4& R) {
    const double a = std::min(w1, w2), b = std::max(w1, w2);
    const double ia = 1.0 / a, ib = 1.0 / b, h = b - a, s = a + b;
    const double is3 = 1.0 / (s * s * s);
    auto split = [](double v, float& hi, float& lo) {
        hi = (float)v;
        lo = (float)(v - (double)hi);
    };
    split(ia, A.x, A.y);
    split(ib, A.z, A.w);
    B = make_float4((float)(ia - ib), (float)is3, (float)(ia * is3), (float)(0.5 * ia * ia * ib / (s * s)));
    k1 = (float)(h * ia * ia * ia * ib * ib / (s * s));
    k2 = (float)(4.0 * ia * ib * is3);
    // the exponential rates log2(e)/a and log2(e)/b as float-float, for the packed path
    float qaHi, qaLo, qbHi, qbLo;
    split(ia * M_LOG2E, qaHi, qaLo);
    split(ib * M_LOG2E, qbHi, qbLo);
    Q = make_float4(-qaHi, qaHi, qaLo, -qbHi);
    R = make_float4(qbHi, qbLo, 0.0f, 0.0f);
}

// Particles with identical parameters of all pair forces form a class; with at most kMaxClasses classes the kernel
// reads the coefficients of a pair from a class-pair table instead of recomputing them (see PairCoef).  Sets the
// class in bits 8..15 of each particle's flags.
constexpr int kMaxClasses = IX_TUNE_PAIR_MAX_CLASSES;
static_assert(kMaxClasses >= 1 && kMaxClasses <= 256, "a particle's class is 8 bits of its flags");

// The class-pair table of one or more systems that share their pair forces' layout (a context, or the systems of a
// batch): flags[s][i] |= class << kClassShift.  Returns the number of classes, 0 when there are more than kMaxClasses
// (then nothing is changed and the kernel takes the per-particle path).
static int classTableHost(const std::vector<const ix_ctx*>& sys, std::vector<std::vector<int>*>& flags,
                          std::vector<PairCoef>& table) {
    std::map<std::vector<double>, int> classes;
    std::vector<std::vector<int>> cls(sys.size());
    std::vector<std::pair<const ix_ctx*, int>> rep;
    for (size_t s = 0; s < sys.size(); s++) {
        const ix_ctx* c = sys[s];
        cls[s].resize(c->n);
        for (int i = 0; i < c->n; i++) {
            std::vector<double> key;
            const int strides[3] = {5, 2, 3};
            for (int t = 0; t < 3; t++)
                if (c->term[t].present)
                    key.insert(key.end(), c->term[t].params.begin() + (size_t)strides[t] * i,
                               c->term[t].params.begin() + (size_t)strides[t] * (i + 1));
            auto it = classes.find(key);
            if (it == classes.end()) {
                if ((int)classes.size() == kMaxClasses) return 0;   // too many classes: per-particle path
                it = classes.emplace(key, (int)classes.size()).first;
                rep.push_back({c, i});
            }
            cls[s][i] = it->second;
        }
    }
    const int T = (int)classes.size();
    table.assign((size_t)T * T, PairCoef{});
    const double beta = sys[0]->term[0].dampingScale;
    for (int ci = 0; ci < T; ci++)
        for (int cj = 0; cj < T; cj++) {
            PairCoef K;
            std::memset(&K, 0, sizeof(K));
            const ix_ctx* ctx = rep[ci].first;   // the classes' parameter layouts are the same in every system
            const int i = rep[ci].second;
            const ix_ctx* ctxJ = rep[cj].first;
            const int j = rep[cj].second;
            if (ctx->term[0].present) {
                const double* p = &ctx->term[0].params[5 * i];
                const double* q = &ctxJ->term[0].params[5 * j];
                double c[3];
                ixhost::xdmCoefficients(p, q, c);
                const double ws = p[4] + q[4];
                K.disp = make_float4((float)c[0], (float)c[1], (float)c[2], ws != 0 ? (float)(2.0 * beta / ws) : 0.0f);
            }
            if (ctx->term[1].present) {
                const double* p = &ctx->term[1].params[2 * i];
                const double* q = &ctxJ->term[1].params[2 * j];
                if (p[1] != 0 && q[1] != 0) overlapCoefficients(p[1], q[1], K.ovA, K.ovB, K.ovC.x, K.ovC.y, K.ovQ, K.ovR);
                K.ovC.z = (float)(p[0] * q[0] / (8.0 * M_PI));
            }
            if (ctx->term[2].present) {
                const double* p = &ctx->term[2].params[3 * i];
                const double* q = &ctxJ->term[2].params[3 * j];
                if (p[2] != 0 && q[2] != 0) overlapCoefficients(p[2], q[2], K.srA, K.srB, K.srC.x, K.srC.y, K.srQ, K.srR);
                const double ws = p[2] + q[2];
                K.srC.z = (float)(ws * ws * ws);
                K.srK = make_float4((float)(0.5 * (p[0] + q[0])), (float)(0.5 * (p[1] + q[1])), 0.0f, 0.0f);
            }
            table[(size_t)ci * T + cj] = K;
        }
    for (size_t s = 0; s < sys.size(); s++)
        for (int i = 0; i < sys[s]->n; i++) (*flags[s])[i] |= cls[s][i] << kClassShift;
    return T;
}

static int buildClassTable(ix_ctx* ctx, std::vector<int>& flags) {
    ctx->P.coef = nullptr;
    ctx->P.numClasses = 0;
    std::vector<const ix_ctx*> sys{ctx};
    std::vector<std::vector<int>*> fl{&flags};
    std::vector<PairCoef> table;
    const int T = classTableHost(sys, fl, table);
    if (T == 0) return IX_OK;
    PairCoef* dTable = nullptr;
    IX_TRY(deviceAlloc(ctx, "classTable", table.size(), &dTable));
    IX_TRY(stageCopy(ctx, dTable, table.data(), table.size() * sizeof(PairCoef)));
    ctx->P.coef = dTable;
    ctx->P.numClasses = T;
    return IX_OK;
}

// The float parameter arrays of a context's pair forces, in its particle order (see PairBuffers) and the flags:
// alchemical bits per term, gate bits, real bit.
static void packPairParams(const ix_ctx* ctx, std::vector<float4>& p0, std::vector<float4>& p1,
                           std::vector<float4>& p2, std::vector<float4>& p3, std::vector<int>& flags) {
    const int n = ctx->n;
    p0.resize(n);
    p1.resize(n);
    p2.resize(n);
    p3.resize(n);
    flags.resize(n);
    for (int i = 0; i < n; i++) {
        float4 a = make_float4(0, 0, 0, 0), b = make_float4(0, 0, 0, 0), c = make_float4(0, 0, 0, 0);
        int f = kFlagReal;
        if (ctx->term[0].present) {
            const double* p = &ctx->term[0].params[5 * i];
            a = make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3]);
            b.x = (float)p[4];
            if (p[3] != 0) f |= kFlagGateDisp;
            if (ctx->term[0].alch[i]) f |= 1;
        }
        double wx = 0, ws = 0;
        if (ctx->term[1].present) {
            const double* p = &ctx->term[1].params[2 * i];
            b.y = (float)p[0];
            wx = p[1];
            c.x = (float)wx;
            c.y = wx != 0 ? (float)(1.0 / wx) : 0.0f;
            if (wx != 0) f |= kFlagGateExch;
            if (ctx->term[1].alch[i]) f |= 2;
        }
        if (ctx->term[2].present) {
            const double* p = &ctx->term[2].params[3 * i];
            b.z = (float)p[0];
            b.w = (float)p[1];
            ws = p[2];
            c.z = (float)ws;
            c.w = ws != 0 ? (float)(1.0 / ws) : 0.0f;
            if (ws != 0) f |= kFlagGateSr;
            if (ctx->term[2].alch[i]) f |= 4;
        }
        p0[i] = a;
        p1[i] = b;
        p2[i] = c;
        flags[i] = f;
        // float remainders of the widths and their reciprocals (float-float values for the kernel)
        const double wide[4] = {wx, wx != 0 ? 1.0 / wx : 0.0, ws, ws != 0 ? 1.0 / ws : 0.0};
        float lo[4];
        for (int k = 0; k < 4; k++) lo[k] = (float)(wide[k] - (double)(float)wide[k]);
        p3[i] = make_float4(lo[0], lo[1], lo[2], lo[3]);
    }
}

static int uploadPairParams(ix_ctx* ctx) {
    const int n = ctx->n;
    std::vector<float4> p0, p1, p2, p3;
    std::vector<int> flags;
    packPairParams(ctx, p0, p1, p2, p3, flags);
    ctx->pairGatesAll = 7u;
    ctx->pairAlchAny = 0u;
    for (int i = 0; i < n; i++) {
        for (int t = 0; t < 3; t++)
            if (!(flags[i] & (kFlagGateDisp << t))) ctx->pairGatesAll &= ~(1u << t);
        ctx->pairAlchAny |= (unsigned)(flags[i] & 7);
    }
    IX_TRY(stageCopy(ctx, ctx->dP0o, p0.data(), n * sizeof(float4)));
    IX_TRY(stageCopy(ctx, ctx->dP1o, p1.data(), n * sizeof(float4)));
    IX_TRY(stageCopy(ctx, ctx->dP2o, p2.data(), n * sizeof(float4)));
    IX_TRY(stageCopy(ctx, ctx->dP3o, p3.data(), n * sizeof(float4)));
    IX_TRY(buildClassTable(ctx, flags));
    IX_TRY(stageCopy(ctx, ctx->dFlagso, flags.data(), n * sizeof(int)));
    IX_TRY(uploadsDone(ctx));
    computeLrc(ctx);
    ctx->pairDirty = false;
    bumpVersion(ctx);
    // a rebuild gathers the parameters into sorted order
    int one = 1;
    IX_TRY(stageCopy(ctx, ctx->L.flag, &one, sizeof(int)));
    return IX_OK;
}

__global__ void kGatherParams(ListBuffers L, const float4* p0o, const float4* p1o, const float4* p2o,
                              const float4* p3o, const int* flagso, float4* p0, float4* p1, float4* p2, float4* p3,
                              int* flags) {
    if (!rebuildRequested(L)) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= L.np) return;
    int i = L.sortedAtom[s];
    if (i >= 0) {
        p0[s] = p0o[i];
        p1[s] = p1o[i];
        p2[s] = p2o[i];
        p3[s] = p3o[i];
        flags[s] = flagso[i];
    }
    else {
        p0[s] = make_float4(0, 0, 0, 0);
        p1[s] = make_float4(0, 0, 0, 0);
        p2[s] = make_float4(0, 0, 0, 0);
        p3[s] = make_float4(0, 0, 0, 0);
        flags[s] = 0;
    }
}

__global__ void kClearFlag(int* flag) { *flag = 0; }

// Estimated number of tiles of the list (the build reports overflows, and the host then grows the buffers).
static long long estimateTiles(const ix_ctx* ctx, int nb) {
    if (ctx->method == IX_NO_CUTOFF) return (long long)nb * (nb + 1) / 2 + nb;
    double volume;
    if (ctx->method == IX_CUTOFF_PERIODIC) volume = ctx->box[0] * ctx->box[4] * ctx->box[8];
    else volume = std::max(1.0, ctx->n / 100.0);   // unknown extent: assume liquid density
    double rho = ctx->n / volume;
    double e = std::cbrt(32.0 / rho);
    double c = ctx->cutoff + kPairSkin;
    double dil = e * e * e + 6 * e * e * c + 3 * M_PI * e * c * c + 4.0 / 3.0 * M_PI * c * c * c;
    double perBlock = std::min<double>(rho * dil, ctx->n) / 32.0 / 2.0 + 2.0;
    long long est = (long long)(1.5 * nb * perBlock) + 64;
    long long full = (long long)nb * (nb + 1) / 2 + nb;
    return std::min(est, full);
}

static int allocatePair(ix_ctx* ctx, long long tileCap) {
    const int n = ctx->n;
    const int nb = (n + 31) / 32, np = nb * 32;
    ListBuffers& L = ctx->L;
    L.n = n;
    L.nb = nb;
    L.np = np;
    // cell grid
    ListGeometry& G = ctx->G;
    G.periodic = ctx->method == IX_CUTOFF_PERIODIC;
    G.useCutoff = ctx->method != IX_NO_CUTOFF;
    G.listCutoff = (float)(ctx->cutoff + kPairSkin);
    int nc[3];
    if (G.periodic) {
        double volume = ctx->box[0] * ctx->box[4] * ctx->box[8];
        double cell = std::cbrt(4.0 * volume / n);
        const double len[3] = {ctx->box[0], ctx->box[4], ctx->box[8]};
        for (int d = 0; d < 3; d++) nc[d] = nearestPow2(len[d] / cell);
    }
    else {
        const int m = nearestPow2(std::cbrt(n / 4.0));
        nc[0] = nc[1] = nc[2] = m;
    }
    for (int d = 0; d < 3; d++) G.nc[d] = nc[d];
    const int numCells = nc[0] * nc[1] * nc[2];
    int bits = 1;
    while ((1 << bits) < std::max(nc[0], std::max(nc[1], nc[2]))) bits++;
    std::vector<std::pair<unsigned long long, int>> order(numCells);
    for (int z = 0; z < nc[2]; z++)
        for (int y = 0; y < nc[1]; y++)
            for (int x = 0; x < nc[0]; x++) {
                int c = (z * nc[1] + y) * nc[0] + x;
                order[c] = {hilbertIndex(x, y, z, bits), c};
            }
    std::sort(order.begin(), order.end());
    std::vector<int> rank(numCells);
    for (int k = 0; k < numCells; k++) rank[order[k].second] = k;
    L.numCells = numCells;

    int* cellRank;
    IX_TRY(deviceAlloc(ctx, "cellRank", numCells, &cellRank));
    IX_TRY(stageCopy(ctx, cellRank, rank.data(), numCells * sizeof(int)));
    L.cellRank = cellRank;
    IX_TRY(deviceAlloc(ctx, "cellKey", n, &L.cellKey));
    IX_TRY(deviceAlloc(ctx, "cellCount", numCells, &L.cellCount));
    IX_TRY(deviceAlloc(ctx, "cellStart", numCells + 1, &L.cellStart));
    IX_TRY(deviceAlloc(ctx, "cellFill", numCells, &L.cellFill));
    IX_TRY(deviceAlloc(ctx, "order", n, &L.order));
    IX_TRY(deviceAlloc(ctx, "bboxMinMax", 8, &L.bboxMinMax));
    IX_TRY(deviceAlloc(ctx, "refPos", 3 * (size_t)n, &L.refPos));
    IX_TRY(deviceAlloc(ctx, "sortedAtom", np, &L.sortedAtom));
    IX_TRY(deviceAlloc(ctx, "slotOf", n, &L.slotOf));
    IX_TRY(deviceAlloc(ctx, "shift", 3 * (size_t)np, &L.shift));
    IX_TRY(deviceAlloc(ctx, "spos", 3 * (size_t)np, &L.spos));
    IX_TRY(deviceAlloc(ctx, "sposf", np, &L.sposf));
    IX_TRY(deviceAlloc(ctx, "bbox", 2 * (size_t)nb, &L.bbox));
    IX_TRY(deviceAlloc(ctx, "blockAtoms", nb, &L.blockAtoms));
    IX_TRY(deviceAlloc(ctx, "blockTiles", nb + 1, &L.blockTiles));
    if (tileCap > (long long)1 << 26) return fail(ctx, IX_ERR_INVALID, "neighbor list too large (%lld tiles)", tileCap);
    ctx->tileCap = (int)tileCap;
    L.tileCap = (int)tileCap;
    IX_TRY(deviceAlloc(ctx, "tileJ", 32 * (size_t)L.tileCap, &L.tileJ));
    IX_TRY(deviceAlloc(ctx, "tileIBlock", L.tileCap, &L.tileIBlock));
    IX_TRY(deviceAlloc(ctx, "tileBucket", L.tileCap, &L.tileBucket));
    IX_TRY(deviceAlloc(ctx, "tileOrder", L.tileCap, &L.tileOrder));
    IX_TRY(deviceAlloc(ctx, "bucketCount", 33, &L.bucketCount));
    IX_TRY(deviceAlloc(ctx, "tileMask", 64 * (size_t)L.tileCap, &L.tileMask));
    IX_TRY(deviceAlloc(ctx, "numTiles", 1, &L.numTiles));
    IX_TRY(deviceAlloc(ctx, "taskCounter", 1, &L.taskCounter));
    IX_TRY(deviceAlloc(ctx, "taskEnergy", 3 * (size_t)L.tileCap, &ctx->dPairPartials));
    IX_CUDA(ctx, cudaMemsetAsync(L.numTiles, 0, sizeof(int), ctx->stream));
    L.flag = ctx->dFlags;
    L.pos = ctx->dPos;
    // exclusions CSR
    std::vector<std::vector<int>> part(n);
    for (auto& e : ctx->exclusions) {
        part[e.first].push_back(e.second);
        part[e.second].push_back(e.first);
    }
    std::vector<int> start(n + 1, 0), list;
    std::vector<int2> range(n);
    for (int i = 0; i < n; i++) {
        std::sort(part[i].begin(), part[i].end());
        start[i] = (int)list.size();
        list.insert(list.end(), part[i].begin(), part[i].end());
        range[i] = part[i].empty() ? make_int2(1, 0) : make_int2(part[i].front(), part[i].back());
    }
    start[n] = (int)list.size();
    int *dStart = nullptr, *dList = nullptr;
    int2* dRange = nullptr;
    IX_TRY(deviceAlloc(ctx, "exclStart", n + 1, &dStart));
    IX_TRY(deviceAlloc(ctx, "exclList", std::max<size_t>(list.size(), 1), &dList));
    IX_TRY(deviceAlloc(ctx, "exclRange", n, &dRange));
    IX_TRY(stageCopy(ctx, dStart, start.data(), (n + 1) * sizeof(int)));
    if (!list.empty())
        IX_TRY(stageCopy(ctx, dList, list.data(), list.size() * sizeof(int)));
    IX_TRY(stageCopy(ctx, dRange, range.data(), n * sizeof(int2)));
    L.exclStart = dStart;
    L.exclList = dList;
    L.exclRange = dRange;
    // parameters
    IX_TRY(deviceAlloc(ctx, "p0o", n, &ctx->dP0o));
    IX_TRY(deviceAlloc(ctx, "p1o", n, &ctx->dP1o));
    IX_TRY(deviceAlloc(ctx, "p2o", n, &ctx->dP2o));
    IX_TRY(deviceAlloc(ctx, "p3o", n, &ctx->dP3o));
    IX_TRY(deviceAlloc(ctx, "p3", np, &ctx->dP3));
    IX_TRY(deviceAlloc(ctx, "flagso", n, &ctx->dFlagso));
    IX_TRY(deviceAlloc(ctx, "p0", np, &ctx->dP0));
    IX_TRY(deviceAlloc(ctx, "p1", np, &ctx->dP1));
    IX_TRY(deviceAlloc(ctx, "p2", np, &ctx->dP2));
    IX_TRY(deviceAlloc(ctx, "flagsSorted", np, &ctx->dFlagsSorted));
    IX_TRY(deviceAlloc(ctx, "forceFixed", 3 * (size_t)np, &ctx->P.forceFixed));
    // accumulators start at zero here; afterwards the kernels that read them clear them
    IX_CUDA(ctx, cudaMemsetAsync(ctx->P.forceFixed, 0, 3 * (size_t)np * sizeof(long long), ctx->stream));
    IX_CUDA(ctx, cudaMemsetAsync(L.taskCounter, 0, sizeof(int), ctx->stream));
    ctx->P.p0 = ctx->dP0;
    ctx->P.p1 = ctx->dP1;
    ctx->P.p2 = ctx->dP2;
    ctx->P.p3 = ctx->dP3;
    ctx->P.flags = ctx->dFlagsSorted;
    L.flags = ctx->dFlagsSorted;
    ctx->P.pairCount = ctx->dCounts;
    int perSM = 0;
    int perSMLean = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kPairTiles<false, false>, 32 * kPairWarps, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSMLean, kPairTiles<true, true>, 32 * kPairWarps, 0);
    ctx->pairGridBlocks = std::max(1, perSM) * ctx->numSMs;
    ctx->pairGridBlocksLean = std::max(1, perSMLean) * ctx->numSMs;
    ctx->P.taskEnergy = ctx->dPairPartials;
    ctx->pairAllocated = true;
    bumpVersion(ctx);
    IX_TRY(uploadPairParams(ctx));
    return IX_OK;
}

static void updateGeometry(ix_ctx* ctx) {
    ListGeometry& G = ctx->G;
    G.box = makeBox(ctx->box);
    G.boxf = makeBoxF(G.box);
}

// ---------------------------------------------------------------------------------------------------------------------
// three-body setup
// ---------------------------------------------------------------------------------------------------------------------

static int allocateAtm(ix_ctx* ctx) {
    const int ns = (int)ctx->siteParams.size() / 3;
    AtmBuffers& A = ctx->A;
    int *dOff, *dPart, *dMol;
    float4* dParams;
    IX_TRY(deviceAlloc(ctx, "siteOffsets", ns + 1, &dOff));
    IX_TRY(deviceAlloc(ctx, "siteParticles", std::max<size_t>(ctx->siteParticles.size(), 1), &dPart));
    IX_TRY(deviceAlloc(ctx, "siteMolecule", ns, &dMol));
    IX_TRY(deviceAlloc(ctx, "siteParams", ns, &dParams));
    IX_TRY(stageCopy(ctx, dOff, ctx->siteOffsets.data(), (ns + 1) * sizeof(int)));
    IX_TRY(stageCopy(ctx, dPart, ctx->siteParticles.data(), ctx->siteParticles.size() * sizeof(int)));
    std::vector<int> mol(ns);
    for (int i = 0; i < ns; i++) mol[i] = ctx->molecule[i] < 0 ? -1 - i : ctx->molecule[i];
    IX_TRY(stageCopy(ctx, dMol, mol.data(), ns * sizeof(int)));
    A.siteOffsets = dOff;
    A.siteParticles = dPart;
    A.molecule = dMol;
    A.siteParams = dParams;
    IX_TRY(deviceAlloc(ctx, "sitePos", 3 * (size_t)ns, &A.sitePos));
    IX_TRY(deviceAlloc(ctx, "siteRef", 3 * (size_t)ns, &A.siteRef));
    IX_TRY(deviceAlloc(ctx, "siteChunkBox", 2 * (size_t)((ns + 31) / 32), &A.chunkBox));
    IX_TRY(deviceAlloc(ctx, "nbrCount", ns, &A.nbrCount));
    IX_TRY(deviceAlloc(ctx, "siteForce", 3 * (size_t)ns, &A.siteForce));
    if (ctx->atmPeriodic) {
        // the cell grid of the list search (its shape follows the box at each evaluation)
        IX_TRY(deviceAlloc(ctx, "siteCellStart", kSiteCellMax + 1, &A.cells.cellStart));
        IX_TRY(deviceAlloc(ctx, "siteCellSites", ns, &A.cells.cellSites));
        IX_TRY(deviceAlloc(ctx, "siteCell", ns, &A.cells.siteCell));
        IX_TRY(deviceAlloc(ctx, "siteWrapped", ns, &A.cells.wrapped));
        // the one-block cell sort scatters up to kSiteSortSharedMax sites in dynamic shared memory (on this device)
        IX_CUDA(ctx, cudaFuncSetAttribute(kSiteCellSort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kSiteSortSharedMax * (int)sizeof(int)));
    }
    {
        // the sites of each particle, so that the finishing kernel gives each particle its share of its sites' forces
        std::vector<int> start(ctx->n + 1, 0), list(ctx->siteParticles.size());
        for (int p : ctx->siteParticles) start[p + 1]++;
        for (int i = 0; i < ctx->n; i++) start[i + 1] += start[i];
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (int sidx = 0; sidx < ns; sidx++)
            for (int k = ctx->siteOffsets[sidx]; k < ctx->siteOffsets[sidx + 1]; k++)
                list[fill[ctx->siteParticles[k]]++] = sidx;
        IX_TRY(deviceAlloc(ctx, "particleSiteStart", (size_t)ctx->n + 1, &ctx->dParticleSiteStart));
        IX_TRY(deviceAlloc(ctx, "particleSites", std::max<size_t>(list.size(), 1), &ctx->dParticleSites));
        IX_TRY(stageCopy(ctx, ctx->dParticleSiteStart, start.data(), start.size() * sizeof(int)));
        IX_TRY(stageCopy(ctx, ctx->dParticleSites, list.data(), list.size() * sizeof(int)));
    }
    IX_TRY(deviceAlloc(ctx, "atmParticleForce", 3 * (size_t)ctx->n, &A.particleForce));
    // accumulators start at zero here; afterwards the kernels that read them clear them
    IX_CUDA(ctx, cudaMemsetAsync(A.siteForce, 0, 3 * (size_t)ns * sizeof(long long), ctx->stream));
    IX_CUDA(ctx, cudaMemsetAsync(A.particleForce, 0, 3 * (size_t)ctx->n * sizeof(long long), ctx->stream));
    // neighbor capacity: twice the expected half list at the site density, at least 64, at most all sites
    if (ctx->atmCap == 0) {
        double volume = ctx->atmPeriodic ? ctx->box[0] * ctx->box[4] * ctx->box[8] : std::max(1.0, ns / 30.0);
        double rho = ns / volume;
        double c = ctx->atmCutoff + kSiteSkin;
        double expect = rho * 4.0 / 3.0 * M_PI * c * c * c / 2.0;
        int cap = (int)std::max(64.0, 2.0 * expect + 32.0);
        cap = std::min(((cap + 31) / 32) * 32, std::max(32, ((ns + 31) / 32) * 32));
        ctx->atmCap = cap;
    }
    A.cap = ctx->atmCap;
    IX_TRY(deviceAlloc(ctx, "nbr", (size_t)ns * A.cap, &A.nbr));
    A.flag = ctx->dFlags + 4;
    A.numParticles = ctx->n;
    // fast kernel: one warp per site; wide kernel (long lists): one wave of blocks over every (site, part) unit
    ctx->atmFastBlocks = std::max(1, (ns + kAtmFastWarps - 1) / kAtmFastWarps);
    ctx->atmGridBlocks = std::max(1, (int)std::min<long long>(((long long)ns * kAtmWideParts + kAtmWarps - 1) / kAtmWarps,
                                                              (long long)ctx->numSMs * 4));
    IX_TRY(deviceAlloc(ctx, "atmPartials", atmPartialCount(ctx), &ctx->dAtmPartials));
    A.energyPartials = ctx->dAtmPartials;
    A.tripleCount = ctx->dCounts + 1;
    ctx->atmAllocated = true;
    ctx->atmDirty = true;
    bumpVersion(ctx);
    return IX_OK;
}

static int uploadAtmParams(ix_ctx* ctx) {
    const int ns = (int)ctx->siteParams.size() / 3;
    std::vector<float4> p(ns);
    for (int i = 0; i < ns; i++)
        p[i] = make_float4((float)ctx->siteParams[3 * i], (float)ctx->siteParams[3 * i + 1],
                           (float)ctx->siteParams[3 * i + 2], ctx->siteAlch[i] ? 1.0f : 0.0f);
    IX_TRY(stageCopy(ctx, (void*)ctx->A.siteParams, p.data(), ns * sizeof(float4)));
    IX_TRY(uploadsDone(ctx));
    int one = 1;
    IX_TRY(stageCopy(ctx, ctx->A.flag, &one, sizeof(int)));
    ctx->atmDirty = false;
    bumpVersion(ctx);
    return IX_OK;
}

// ---------------------------------------------------------------------------------------------------------------------
// evaluation
// ---------------------------------------------------------------------------------------------------------------------

// The accumulators are read and cleared here, so the next evaluation starts from zero without memsets (they are
// zeroed once when allocated).
__global__ void kFinalize(int n, int np, const int* slotOf, long long* pairForce, long long* atmForce,
                          double* outForces, long long* addFixed, int stride) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        long long f[3] = {0, 0, 0};
        if (pairForce) {
            int s = slotOf[i];
            for (int d = 0; d < 3; d++) {
                f[d] = pairForce[d * np + s];
                pairForce[d * np + s] = 0;
            }
        }
        if (atmForce) {
            for (int d = 0; d < 3; d++) {
                f[d] += atmForce[d * n + i];
                atmForce[d * n + i] = 0;
            }
        }
        if (outForces) {
            const double inv = 1.0 / kFixedScale;
            outForces[3 * i] = (double)f[0] * inv;
            outForces[3 * i + 1] = (double)f[1] * inv;
            outForces[3 * i + 2] = (double)f[2] * inv;
        }
        if (addFixed) {
            atomicAddFixed(addFixed + i, f[0]);
            atomicAddFixed(addFixed + stride + i, f[1]);
            atomicAddFixed(addFixed + 2 * stride + i, f[2]);
        }
    }
}

// Term energies from the per-tile / per-warp partials: each block sums a fixed share, then the last block adds the
// block sums in order, so the result is identical on every run.  lrcEnergy (the long range correction, from the host)
// joins term 0.  The last block also publishes the interaction counts (counts[0..1] -> counts[2..3], clearing the
// accumulators) and resets the pair kernel's tile counter for the next evaluation.
constexpr int kReduceBlocks = 64;

struct EnergyReduction {
    const double* pairPartials;          // null: no pair terms
    const int* numPairPartials;
    int pairCap;
    const double* atmPartials;           // null: no three-body term
    int numAtmWarps;
    double lrcEnergy;
    double* outEnergy;
    double* blockSums;
    unsigned* ticket;
    unsigned long long* counts;
    int* taskCounter;
};

// One block (of `numBlocks`) of the energy reduction; 256 threads.
__device__ void reduceEnergiesBlock(const EnergyReduction& R, int block, int numBlocks) {
    __shared__ double red[4][256];
    __shared__ bool last;
    const int t = threadIdx.x;
    // each block sums a fixed contiguous share of each array; the last block to finish adds the block sums in order
    auto share = [&](int total, int& lo, int& hi) {
        const int per = (total + numBlocks - 1) / numBlocks;
        lo = min(block * per, total);
        hi = min(lo + per, total);
    };
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    int lo, hi;
    if (R.pairPartials) {
        share(min(*R.numPairPartials, R.pairCap), lo, hi);
        for (int w = lo + t; w < hi; w += 256)
            for (int k = 0; k < 3; k++) s[k] += R.pairPartials[3 * w + k];
    }
    if (R.atmPartials) {
        share(R.numAtmWarps, lo, hi);
        for (int w = lo + t; w < hi; w += 256) s[3] += R.atmPartials[w];
    }
    for (int k = 0; k < 4; k++) red[k][t] = s[k];
    __syncthreads();
    for (int half = 128; half > 0; half >>= 1) {
        if (t < half)
            for (int k = 0; k < 4; k++) red[k][t] += red[k][t + half];
        __syncthreads();
    }
    if (t == 0) {
        for (int k = 0; k < 4; k++) R.blockSums[4 * block + k] = red[k][0];
        __threadfence();
        // wraps to 0 on the last block, ready for the next launch
        last = atomicInc(R.ticket, numBlocks - 1) == (unsigned)(numBlocks - 1);
    }
    __syncthreads();
    if (!last) return;
    // the block sums are loaded in parallel, then added in block order
    __threadfence();
    for (int k = t; k < 4 * numBlocks; k += 256) red[k & 3][k >> 2] = ((volatile double*)R.blockSums)[k];
    __syncthreads();
    if (t < 4) {
        double v = 0.0;
        for (int b = 0; b < numBlocks; b++) v += red[t][b];
        if (t == 0) v += R.lrcEnergy;
        if (R.outEnergy) R.outEnergy[t] = v;
        if (t == 0) {
            if (R.counts) {
                R.counts[2] = R.counts[0];
                R.counts[3] = R.counts[1];
                R.counts[0] = 0;
                R.counts[1] = 0;
            }
            if (R.taskCounter) *R.taskCounter = 0;
        }
    }
}

__global__ void kReduceEnergies(const double* pairPartials, const int* numPairPartials, int pairCap,
                                const double* atmPartials, int numAtmWarps, double lrcEnergy, double* outEnergy,
                                double* blockSums, unsigned* ticket, unsigned long long* counts, int* taskCounter) {
    const EnergyReduction R{pairPartials, numPairPartials, pairCap, atmPartials, numAtmWarps, lrcEnergy,
                            outEnergy,    blockSums,       ticket,  counts,      taskCounter};
    reduceEnergiesBlock(R, blockIdx.x, gridDim.x);
}

struct FinishForces {
    int n, np;
    const int* slotOf;
    long long* pairForce;                // null: no pair terms; cleared as read
    const long long* siteForce;          // null: no three-body term (cleared by the next evaluation's centroid kernel)
    int numSites;
    const int* siteOffsets;
    const int* particleSiteStart;
    const int* particleSites;
    double* outForces;
    long long* addFixed;
    int stride;
    const int* addSlot;                  // row of each particle in addFixed (null: its index)
    const double* invMass;               // null: no velocity half kick
    double* vel;
    double halfDt;
    int blocks;                          // blocks of 256 particles; the grid's remaining blocks reduce the energies
};

// The end of an evaluation in one launch: each particle's force (its pair force and its share of the forces on its
// three-body sites, in 64-bit fixed point, so the sum is the same in any order) to the outputs, and in an MD step
// the second velocity half kick; the grid's last kReduceBlocks blocks reduce the term energies.
__global__ void kFinish(FinishForces F, EnergyReduction R) {
    if ((int)blockIdx.x >= F.blocks) {
        reduceEnergiesBlock(R, (int)blockIdx.x - F.blocks, (int)gridDim.x - F.blocks);
        return;
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.n) return;
    long long f[3] = {0, 0, 0};
    if (F.pairForce) {
        const int s = F.slotOf[i];
        for (int d = 0; d < 3; d++) {
            f[d] = F.pairForce[d * F.np + s];
            F.pairForce[d * F.np + s] = 0;
        }
    }
    if (F.siteForce)
        for (int k = F.particleSiteStart[i]; k < F.particleSiteStart[i + 1]; k++) {
            const int site = F.particleSites[k];
            const double inv = 1.0 / (double)(F.siteOffsets[site + 1] - F.siteOffsets[site]);
            for (int d = 0; d < 3; d++) {
                const long long v = F.siteForce[d * F.numSites + site];
                if (v != 0) f[d] += __double2ll_rn((double)v * inv);
            }
        }
    const double inv = 1.0 / kFixedScale;
    const double fx = (double)f[0] * inv, fy = (double)f[1] * inv, fz = (double)f[2] * inv;
    if (F.outForces) {
        F.outForces[3 * i] = fx;
        F.outForces[3 * i + 1] = fy;
        F.outForces[3 * i + 2] = fz;
    }
    if (F.addFixed) {
        // a slot map that did not name this particle (not a permutation) leaves it out rather than write elsewhere
        const int row = F.addSlot ? F.addSlot[i] : i;
        if (row >= 0 && row < F.stride) {
            atomicAddFixed(F.addFixed + row, f[0]);
            atomicAddFixed(F.addFixed + F.stride + row, f[1]);
            atomicAddFixed(F.addFixed + 2 * F.stride + row, f[2]);
        }
    }
    if (F.invMass) {
        const double h = F.halfDt * F.invMass[i];
        F.vel[3 * i] += h * fx;
        F.vel[3 * i + 1] += h * fy;
        F.vel[3 * i + 2] += h * fz;
    }
}

// The start of an MD step over the pair list's sorted slots, in one launch: the first velocity half kick and the
// drift of each particle, the displacement check that requests a list rebuild, and the refresh of its sorted
// position (the rebuild, when it runs, sorts and refreshes again).
__global__ void kStepStart(ListBuffers L, double* pos, double dt, const double* invMass, const double* force,
                           double* vel, float maxMove2) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    if (s < L.n) {
        const int i = L.sortedAtom[s];
        const double h = 0.5 * dt * invMass[i];
        double x[3];
        for (int d = 0; d < 3; d++) {
            const double v = vel[3 * i + d] + h * force[3 * i + d];
            vel[3 * i + d] = v;
            x[d] = pos[3 * i + d] + dt * v;
            pos[3 * i + d] = x[d];
        }
        const double dx = x[0] - L.refPos[3 * i], dy = x[1] - L.refPos[3 * i + 1], dz = x[2] - L.refPos[3 * i + 2];
        moved = (float)(dx * dx + dy * dy + dz * dz) > maxMove2;
        const double sx = x[0] - L.shift[3 * s], sy = x[1] - L.shift[3 * s + 1], sz = x[2] - L.shift[3 * s + 2];
        L.spos[3 * s] = sx;
        L.spos[3 * s + 1] = sy;
        L.spos[3 * s + 2] = sz;
        L.sposf[s] = make_float4((float)sx, (float)sy, (float)sz, 0.0f);
    }
    if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) atomicOr(L.flag, 1);
}

// Which terms of the context are selected by a force-group mask.
static unsigned selectedTerms(const ix_ctx* ctx, int groups) {
    unsigned mask = 0;
    for (int t = 0; t < 3; t++)
        if (ctx->term[t].present && ((groups >> ctx->term[t].group) & 1)) mask |= 1u << t;
    if (ctx->atmPresent && ((groups >> ctx->atmGroup) & 1)) mask |= 8u;
    return mask;
}

static PairTermConfig pairConfig(const ix_ctx* ctx, unsigned terms) {
    PairTermConfig C{};
    C.termMask = (int)(terms & 7u);
    for (int t = 0; t < 3; t++) {
        const PairTerm& T = ctx->term[t];
        double lam = lambdaOf(ctx, T.alchName, T.anyAlch);
        C.lambda[t] = (float)lam;
        C.softShift[t] = (T.anyAlch && T.softcoreRadius > 0) ? (float)((1.0 - lam) * std::pow(T.softcoreRadius, 6.0)) : 0.0f;
        C.useSwitch[t] = T.useSwitch;
        C.switchDist[t] = (float)T.switchDistance;
        C.invSwitchWidth[t] = T.useSwitch ? (float)(1.0 / (ctx->cutoff - T.switchDistance)) : 0.0f;
        C.overlapMethod[t] = T.overlapMethod;
    }
    C.twoBeta = (float)(2.0 * ctx->term[0].dampingScale);
    // the exchange and short-range terms share one overlap when their widths and methods agree for every particle
    if (ctx->pairShareOverlap < 0) {
        bool same = ctx->term[1].present && ctx->term[2].present;
        for (int i = 0; i < ctx->n && same; i++) same = ctx->term[1].params[2 * i + 1] == ctx->term[2].params[3 * i + 2];
        ctx->pairShareOverlap = same;
    }
    C.shareOverlap = ctx->pairShareOverlap && ctx->term[1].overlapMethod == ctx->term[2].overlapMethod;
    C.useCutoff = ctx->method != IX_NO_CUTOFF;
    C.periodic = ctx->method == IX_CUTOFF_PERIODIC;
    C.cutoff = ctx->cutoff;
    C.cutoff2 = (float)(ctx->cutoff * ctx->cutoff);
    C.box = ctx->G.box;
    for (int k = 0; k < 3; k++) {
        const double v[3] = {C.box.a[k], C.box.b[k], C.box.c[k]};
        float* hi[3] = {C.boxff.a, C.boxff.b, C.boxff.c};
        float* lo[3] = {C.boxff.aLo, C.boxff.bLo, C.boxff.cLo};
        for (int m = 0; m < 3; m++) {
            hi[m][k] = (float)v[m];
            lo[m][k] = (float)(v[m] - (double)hi[m][k]);
        }
        C.boxff.inv[k] = (float)C.box.inv[k];
    }
    C.boxff.triclinic = C.box.triclinic;
    return C;
}

static int stageUploads(ix_ctx* ctx, unsigned terms);

__global__ void kSetCondition(cudaGraphConditionalHandle handle, const int* flag) {
    cudaGraphSetConditional(handle, *(volatile const int*)flag != 0 ? 1u : 0u);
}

// Profiling events: while capturing, external event-record nodes of the graph; launched directly, ordinary records.
static void recordTiming(ix_ctx* ctx, int i, cudaStream_t s) {
    if (!ctx->profiling) return;
    if (ctx->capturing) cudaEventRecordWithFlags(ctx->ev[i], s, cudaEventRecordExternal);
    else cudaEventRecord(ctx->ev[i], s);
}

__global__ void kClearFlagIf(int* target, const int* gate) {
    if (*(volatile const int*)gate != 0) *target = 0;
}

// Launch `body` (a callable taking the stream to launch on) when *flag is set, else `orElse` (size 2) or nothing.
// While the evaluation is being captured into a graph this is a conditional node whose branches are captured on the
// context's third stream; the flag is read on the device each time the graph runs, so a step without a list rebuild
// launches none of the rebuild kernels.  Launched directly, `body` runs, its kernels reading the flag themselves
// (and `body` containing `orElse`'s work).  The launch counter keeps the kernels of the branch taken when the flag
// is clear.
template <class Body, class Else>
static int launchConditional(ix_ctx* ctx, cudaStream_t st, const int* flag, Body body, Else orElse, int size) {
    if (!ctx->capturing) return body(st);
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t numDeps = 0;
    IX_CUDA(ctx, cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &numDeps));
    cudaGraphConditionalHandle handle;
    IX_CUDA(ctx, cudaGraphConditionalHandleCreate(&handle, graph, 0, cudaGraphCondAssignDefault));
    kSetCondition<<<1, 1, 0, st>>>(handle, flag);
    ctx->launches += 1;
    IX_CUDA(ctx, cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &numDeps));
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeIf;
    params.conditional.size = (unsigned)size;
    cudaGraphNode_t node;
    IX_CUDA(ctx, cudaGraphAddNode(&node, graph, deps, numDeps, &params));
    for (int k = 0; k < size; k++) {
        IX_CUDA(ctx, cudaStreamBeginCaptureToGraph(ctx->streamBody, params.conditional.phGraph_out[k], nullptr,
                                                   nullptr, 0, cudaStreamCaptureModeThreadLocal));
        const long long before = ctx->launches;
        const int rc = k == 0 ? body(ctx->streamBody) : orElse(ctx->streamBody);
        cudaGraph_t captured = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ctx->streamBody, &captured);
        if (k == 0) ctx->launches = before;
        if (rc != IX_OK) return rc;
        IX_CUDA(ctx, e);
    }
    IX_CUDA(ctx, cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return IX_OK;
}

template <class Body>
static int launchIf(ix_ctx* ctx, cudaStream_t st, const int* flag, Body body) {
    return launchConditional(ctx, st, flag, body, body, 1);
}

template <class Body, class Else>
static int launchIfElse(ix_ctx* ctx, cudaStream_t st, const int* flag, Body body, Else orElse) {
    return launchConditional(ctx, st, flag, body, orElse, 2);
}

// Launch the whole evaluation on the context's stream.  Forces go to outForces (device, n x 3 doubles) and/or are
// added to addFixed; energies to outEnergy (device, 4 doubles).
// The second velocity half kick of an MD step, done by the evaluation's finishing kernel.
struct StepKick {
    const double* invMass;
    double* vel;
    double halfDt;
    bool started = true;     // the step's first kernel checked the displacement and refreshed the sorted positions
};

// `kick`: an MD step whose first kernel (kStepStart) has already moved the particles, checked their displacement and
// refreshed the pair list's sorted positions; the evaluation ends with the second half kick.
static int launchEvaluation(ix_ctx* ctx, unsigned terms, double* outForces, double* outEnergy, long long* addFixed,
                            int stride, const StepKick* kick = nullptr, const int* addSlot = nullptr) {
    const int n = ctx->n;
    cudaStream_t st = ctx->stream;
    const bool doPair = (terms & 7u) != 0;
    const bool doAtm = (terms & 8u) != 0;
    IX_TRY(stageUploads(ctx, terms));
    // the three-body chain runs on a second stream, concurrently with the pair list and pair kernel
    const bool fork = doPair && doAtm && !ctx->serialize;
    cudaStream_t sa = fork ? ctx->stream2 : st;
    if (fork) {
        IX_CUDA(ctx, cudaEventRecord(ctx->evFork, st));
        IX_CUDA(ctx, cudaStreamWaitEvent(sa, ctx->evFork, 0));
    }
    if (doAtm) {
        AtmBuffers& A = ctx->A;
        AtmConfig C{};
        C.numSites = (int)ctx->siteParams.size() / 3;
        C.periodic = ctx->atmPeriodic;
        C.box = makeBox(ctx->box);
        C.boxf = makeBoxF(C.box);
        C.cutoff2 = (float)(ctx->atmCutoff * ctx->atmCutoff);
        double lc = ctx->atmCutoff + kSiteSkin;
        C.listCutoff2 = (float)(lc * lc);
        C.scale = (float)ctx->atmScale;
        C.lambda = (float)lambdaOf(ctx, ctx->atmAlchName, ctx->atmAnyAlch);
        C.useTangToennies = ctx->atmDamping == IX_TANG_TOENNIES;
        C.twoBeta = (float)(2.0 * ctx->atmDampingScale);
        C.invCentroidRadius = ctx->atmCentroidRadius > 0 ? (float)(1.0 / ctx->atmCentroidRadius) : 0.0f;
        C.maxMove2 = 0.25f * kSiteSkin * kSiteSkin;
        const int tpb = 256;
        const int gS = (C.numSites + 63) / 64;   // 64-thread blocks, so that a few thousand sites reach every SM
        // the wide kernel's energy slots start at zero (it runs only while some list is long)
        C.zeroSlots = ctx->atmGridBlocks * kAtmWarps;
        C.zeroOffset = ctx->atmFastBlocks * kAtmFastWarps;
        // the cell grid of the list search in a rectangular periodic box with at least three cells per edge
        A.cells.nc[0] = A.cells.nc[1] = A.cells.nc[2] = 0;
        if (C.periodic && !C.box.triclinic && A.cells.cellStart) {
            const double width = ctx->atmCutoff + kSiteSkin + 1e-3;   // room for the float rounding of the binning
            const double len[3] = {ctx->box[0], ctx->box[4], ctx->box[8]};
            int nc[3];
            for (int d = 0; d < 3; d++) nc[d] = (int)std::floor(len[d] / width);
            if (nc[0] >= 3 && nc[1] >= 3 && nc[2] >= 3 && (long long)nc[0] * nc[1] * nc[2] <= kSiteCellMax)
                for (int d = 0; d < 3; d++) {
                    A.cells.nc[d] = nc[d];
                    A.cells.cellsPerNm[d] = (float)(nc[d] / len[d]);
                }
        }
        kSiteCentroids<<<gS, 64, 0, sa>>>(A, C, ctx->dPos);
        // site list rebuild when the centroid kernel set the flag: these kernels return at once otherwise (short
        // launches cost less than a conditional graph node); the long-list flag is recomputed with the lists
        kClearFlagIf<<<1, 1, 0, sa>>>(A.flag + 2, A.flag);
        if (A.cells.nc[0]) {
            const int sharedSites = C.numSites <= kSiteSortSharedMax;
            kSiteCellSort<<<1, 1024, sharedSites ? C.numSites * sizeof(int) : 0, sa>>>(A, C, sharedSites);
            kSiteNeighborsCells<<<(C.numSites * 32 + tpb - 1) / tpb, tpb, 0, sa>>>(A, C);
            ctx->launches += 1;
        }
        else kSiteNeighbors<<<(C.numSites * 32 + tpb - 1) / tpb, tpb, 0, sa>>>(A, C);
        kClearFlag<<<1, 1, 0, sa>>>(A.flag);
        recordTiming(ctx, 2, sa);
        kTriplesFast<<<ctx->atmFastBlocks, 32 * kAtmFastWarps, 0, sa>>>(A, C);
        // the sites whose lists are too long for the fast kernel: the kernel returns at once when there are none
        kTriplesWide<<<ctx->atmGridBlocks, 32 * kAtmWarps, sizeof(AtmWarpStorage) * kAtmWarps, sa>>>(
            A, C, ctx->atmFastBlocks * kAtmFastWarps, A.flag + 2);
        ctx->launches += 6;
        recordTiming(ctx, 3, sa);
        ctx->evAtm = ctx->profiling;
        IX_CUDA(ctx, cudaGetLastError());
    }
    double lrcEnergy = 0.0;
    if (doPair) {
        ListBuffers& L = ctx->L;
        const int tpb = 256;
        const int gN = (n + tpb - 1) / tpb, gNp = (L.np + tpb - 1) / tpb;
        const int gCells = (L.numCells + tpb - 1) / tpb;
        const bool stepStarted = kick != nullptr && kick->started;
        if (!stepStarted) {
            kCheckDisplacement<<<gN, tpb, 0, st>>>(L, 0.25f * kPairSkin * kPairSkin);
            ctx->launches += 1;
        }
        // the current positions in the build frame, every step
        auto refresh = [&](cudaStream_t s) {
            kUpdateSortedPositions<<<gNp, tpb, 0, s>>>(L);
            ctx->launches += 1;
            return IX_OK;
        };
        // list rebuild (the displacement check set the flag): cell sort, then the tiles and their masks from the
        // refreshed positions
        auto rebuild = [&](cudaStream_t s) {
            kResetCells<<<std::max(1, std::min(gCells, 1024)), tpb, 0, s>>>(L);
            if (!ctx->G.periodic) kParticleBounds<<<gN, tpb, 0, s>>>(L);
            kCellKeys<<<gN, tpb, 0, s>>>(L, ctx->G);
            kScanCells<<<1, 1024, 0, s>>>(L);
            kScatterCells<<<gN, tpb, 0, s>>>(L);
            kSortWithinCells<<<gCells, tpb, 0, s>>>(L);
            kSortedAtoms<<<gNp, tpb, 0, s>>>(L, ctx->G);
            kGatherParams<<<gNp, tpb, 0, s>>>(L, ctx->dP0o, ctx->dP1o, ctx->dP2o, ctx->dP3o, ctx->dFlagso, ctx->dP0,
                                              ctx->dP1, ctx->dP2, ctx->dP3, ctx->dFlagsSorted);
            refresh(s);
            kBlockBounds<<<(L.nb * 32 + tpb - 1) / tpb, tpb, 0, s>>>(L, ctx->G);
            kListTiles<0><<<L.nb, kListThreads, 0, s>>>(L, ctx->G);
            kScanTiles<<<1, 1024, 0, s>>>(L);
            kListTiles<1><<<L.nb, kListThreads, 0, s>>>(L, ctx->G);
            // grids no larger than the tiles need, so that a small system's launches leave the other SMs to the
            // kernels of other streams
            kTileMasks<<<std::min(ctx->numSMs * 8, std::max(1, (L.tileCap + kListWarps - 1) / kListWarps)), kListThreads,
                         0, s>>>(L, ctx->G);
            kTileOrder<<<std::min(ctx->numSMs, std::max(1, (L.tileCap + 255) / 256)), 256, 0, s>>>(L);
            kClearFlag<<<1, 1, 0, s>>>(L.flag);
            ctx->launches += ctx->G.periodic ? 14 : 15;
            return IX_OK;
        };
        if (stepStarted) IX_TRY(launchIf(ctx, st, L.flag, rebuild));
        else IX_TRY(launchIfElse(ctx, st, L.flag, rebuild, refresh));
        PairTermConfig C = pairConfig(ctx, terms);
        // the lean instantiation when no selected term has a soft core, a switching function or the order-2 overlap
        bool lean = true;
        for (int t = 0; t < 3; t++)
            if ((terms >> t) & 1u) lean = lean && C.softShift[t] == 0.0f && !C.useSwitch[t] && C.overlapMethod[t] == 0;
        recordTiming(ctx, 0, st);
        // the class-pair table serves the exact overlap method only
        bool table = ctx->P.coef != nullptr;
        for (int t = 1; t < 3; t++)
            if ((terms >> t) & 1u) table = table && C.overlapMethod[t] == 0;
        // a persistent grid, but no more warps than tiles (a small system leaves the other SMs to other streams)
        const int grid = std::min(lean ? ctx->pairGridBlocksLean : ctx->pairGridBlocks,
                                  std::max(1, (L.tileCap + kPairWarps - 1) / kPairWarps));
        // every pair of every selected term evaluated unscaled: no per-pair gate or scale tests
        bool uniform = lean;
        for (int t = 0; t < 3; t++)
            if ((terms >> t) & 1u)
                uniform = uniform && ((ctx->pairGatesAll >> t) & 1u) &&
                          (!((ctx->pairAlchAny >> t) & 1u) || C.lambda[t] == 1.0f);
        // a small class-pair table is staged in shared memory by each block
        PairBuffers P = ctx->P;
        const size_t tableBytes = (size_t)P.numClasses * P.numClasses * sizeof(PairCoef);
        const size_t dyn = table && tableBytes <= (size_t)IX_TUNE_PAIR_SHARED_TABLE_BYTES ? tableBytes : 0;
        P.coefShared = dyn > 0;
        C.coefShared = P.coefShared;
        if (lean && table && uniform) kPairTiles<true, true, true><<<grid, 32 * kPairWarps, dyn, st>>>(L, P, C);
        else if (lean && uniform) kPairTiles<true, false, true><<<grid, 32 * kPairWarps, 0, st>>>(L, P, C);
        else if (lean && table) kPairTiles<true, true><<<grid, 32 * kPairWarps, dyn, st>>>(L, P, C);
        else if (lean) kPairTiles<true, false><<<grid, 32 * kPairWarps, 0, st>>>(L, P, C);
        else if (table) kPairTiles<false, true><<<grid, 32 * kPairWarps, dyn, st>>>(L, P, C);
        else kPairTiles<false, false><<<grid, 32 * kPairWarps, 0, st>>>(L, P, C);
        ctx->launches += 1;
        recordTiming(ctx, 1, st);
        ctx->evPair = ctx->profiling;
        IX_CUDA(ctx, cudaGetLastError());
        const PairTerm& D = ctx->term[0];
        if ((terms & 1u) && (D.lrcCoef != 0 || D.lrcAlchCoef != 0)) {
            double lam = lambdaOf(ctx, D.alchName, D.anyAlch);
            lrcEnergy = (D.lrcCoef + lam * D.lrcAlchCoef) / (ctx->box[0] * ctx->box[4] * ctx->box[8]);
        }
    }
    if (fork) {
        IX_CUDA(ctx, cudaEventRecord(ctx->evJoin, sa));
        IX_CUDA(ctx, cudaStreamWaitEvent(st, ctx->evJoin, 0));
    }
    FinishForces F{};
    F.n = n;
    F.np = ctx->L.np;
    F.slotOf = ctx->L.slotOf;
    F.pairForce = doPair ? ctx->P.forceFixed : nullptr;
    F.siteForce = doAtm ? ctx->A.siteForce : nullptr;
    F.numSites = (int)ctx->siteParams.size() / 3;
    F.siteOffsets = ctx->A.siteOffsets;
    F.particleSiteStart = ctx->dParticleSiteStart;
    F.particleSites = ctx->dParticleSites;
    F.outForces = outForces;
    F.addFixed = addFixed;
    F.stride = stride;
    F.addSlot = addSlot;
    if (kick) {
        F.invMass = kick->invMass;
        F.vel = kick->vel;
        F.halfDt = kick->halfDt;
    }
    F.blocks = (n + 255) / 256;
    EnergyReduction R{doPair ? ctx->dPairPartials : nullptr, ctx->L.numTiles, ctx->L.tileCap,
                      doAtm ? ctx->dAtmPartials : nullptr, (int)atmPartialCount(ctx), lrcEnergy, outEnergy,
                      ctx->dEnergyBlocks, ctx->dReduceTicket, ctx->dCounts, doPair ? ctx->L.taskCounter : nullptr};
    kFinish<<<F.blocks + kReduceBlocks, 256, 0, st>>>(F, R);
    ctx->launches += 1;
    IX_CUDA(ctx, cudaGetLastError());
    return IX_OK;
}

// Make sure buffers exist for the selected terms.
static int prepare(ix_ctx* ctx, unsigned terms) {
    if (!ctx->havePositions) return fail(ctx, IX_ERR_STATE, "positions have not been set");
    if ((terms & 7u) && !ctx->pairAllocated) {
        updateGeometry(ctx);
        const int nb = (ctx->n + 31) / 32;
        IX_TRY(allocatePair(ctx, ctx->tileCapRequest > 0 ? ctx->tileCapRequest : estimateTiles(ctx, nb)));
    }
    if ((terms & 8u) && !ctx->atmAllocated) IX_TRY(allocateAtm(ctx));
    return IX_OK;
}

// After a synchronized evaluation: grow the lists that overflowed.  Returns true if the evaluation must be redone.
static int checkOverflowFlags(ix_ctx* ctx, unsigned terms, const int* flags, bool& redo);

static int checkOverflow(ix_ctx* ctx, unsigned terms, bool& redo) {
    int flags[6];
    IX_CUDA(ctx, cudaMemcpy(flags, ctx->dFlags, sizeof(flags), cudaMemcpyDeviceToHost));
    return checkOverflowFlags(ctx, terms, flags, redo);
}

// The same from flags already copied to the host (6 ints from ctx->dFlags).
static int checkOverflowFlags(ix_ctx* ctx, unsigned terms, const int* flags, bool& redo) {
    NvtxRange nvtxRange("list overflow check");
    redo = false;
    if ((terms & 7u) && flags[1]) {
        long long tiles = 0;
        int cnt = 0;
        IX_CUDA(ctx, cudaMemcpy(&cnt, ctx->L.blockTiles + ctx->L.nb, sizeof(int), cudaMemcpyDeviceToHost));
        tiles = std::max<long long>(2LL * ctx->tileCap, (long long)(1.3 * cnt) + 64);
        int zero[4] = {1, 0, 0, 0};
        IX_CUDA(ctx, cudaMemcpy(ctx->dFlags, zero, sizeof(zero), cudaMemcpyHostToDevice));
        ctx->pairAllocated = false;
        IX_TRY(allocatePair(ctx, tiles));
        redo = true;
        bumpVersion(ctx);
    }
    if ((terms & 8u) && flags[5]) {
        // the sites whose lists overflowed were evaluated by scanning every later site, so the results stand; the
        // lists grow for the next evaluations
        int cap = 0;
        {
            std::vector<int> counts(ctx->siteParams.size() / 3);
            IX_CUDA(ctx, cudaMemcpy(counts.data(), ctx->A.nbrCount, counts.size() * sizeof(int),
                                    cudaMemcpyDeviceToHost));
            for (int c : counts) cap = std::max(cap, c);
        }
        const int allSites = (((int)ctx->siteParams.size() / 3 + 31) / 32) * 32 + 32;
        ctx->atmCap = std::min(std::max(2 * ctx->atmCap, ((cap * 5 / 4 + 31) / 32) * 32), allSites);
        int f[2] = {1, 0};
        IX_CUDA(ctx, cudaMemcpy(ctx->dFlags + 4, f, sizeof(f), cudaMemcpyHostToDevice));
        IX_TRY(allocateAtm(ctx));
        IX_TRY(uploadAtmParams(ctx));
        bumpVersion(ctx);
    }
    return IX_OK;
}

// The uploads launchEvaluation would otherwise start itself.  They synchronize, so they run before a capture.
static int stageUploads(ix_ctx* ctx, unsigned terms) {
    updateGeometry(ctx);
    if ((terms & 7u) && ctx->pairDirty) IX_TRY(uploadPairParams(ctx));
    if ((terms & 8u) && ctx->atmDirty) IX_TRY(uploadAtmParams(ctx));
    return IX_OK;
}

// Enqueue work on the context's stream through a cached CUDA graph: captured on first use and again after a change of
// state (ctx->version) or of the key, otherwise replayed with one launch.  enqueue() must not synchronize.
template <class F>
static int launchGraph(ix_ctx* ctx, LaunchGraph& g, const GraphKey& key, F&& enqueue) {
    if (!ctx->useGraphs) return enqueue();
    if (!g.exec || g.version != ctx->version || !(g.key == key)) {
        const long long before = ctx->launches;
        NvtxRange nvtxRange("graph capture");
        IX_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        ctx->capturing = true;
        const int rc = enqueue();
        ctx->capturing = false;
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        if (rc != IX_OK || e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            ctx->launches = before;
            if (rc != IX_OK) return rc;
            return fail(ctx, IX_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
        }
        // a new instantiation (the conditional nodes' handles belong to the captured graph)
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
        {
            const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
            if (ie != cudaSuccess) {
                cudaGraphDestroy(graph);
                g.exec = nullptr;
                ctx->launches = before;
                return fail(ctx, IX_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(ie));
            }
        }
        cudaGraphDestroy(graph);
        g.launches = ctx->launches - before;
        ctx->launches = before;
        g.key = key;
        g.version = ctx->version;
    }
    IX_CUDA(ctx, cudaGraphLaunch(g.exec, ctx->stream));
    ctx->launches += g.launches;
    return IX_OK;
}

static void releaseGraph(LaunchGraph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
}

// ---------------------------------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------------------------------

// The status block of a context (device, and a pinned host copy): flags (8 ints), term energies (4 doubles), counts
// (4 unsigned long long).
constexpr size_t kStatusBytes = 96;

// Pinned host slots of 128 bytes for the status copies, carved from shared pinned pages (one cudaHostAlloc per
// 64 KB); the pages live until the process exits.
struct PinnedSlots {
    std::mutex m;
    std::vector<unsigned char*> free;
    unsigned char* take() {
        std::lock_guard<std::mutex> lock(m);
        if (free.empty()) {
            unsigned char* page = nullptr;
            if (cudaHostAlloc(reinterpret_cast<void**>(&page), size_t(64) << 10, cudaHostAllocDefault) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            for (size_t off = 0; off + 128 <= (size_t(64) << 10); off += 128) free.push_back(page + off);
        }
        unsigned char* p = free.back();
        free.pop_back();
        return p;
    }
    void give(unsigned char* p) {
        std::lock_guard<std::mutex> lock(m);
        free.push_back(p);
    }
};

static PinnedSlots& pinnedSlots() {
    static PinnedSlots* slots = new PinnedSlots();
    return *slots;
}

// The device side of a context: streams, events and the buffers every evaluation uses (through ctx->arena when a
// server owns the context).  A context described on the host only (a server request) gets it on admission.
static int ctxInitDevice(ix_ctx* ctx) {
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    IX_CUDA(ctx, cudaDeviceGetAttribute(&ctx->numSMs, cudaDevAttrMultiProcessorCount, ctx->device));
    // streams and events a server hands over from its pool are kept
    if ((!ctx->stream && cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) ||
        (!ctx->stream2 && cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking) != cudaSuccess) ||
        (!ctx->streamBody && cudaStreamCreateWithFlags(&ctx->streamBody, cudaStreamNonBlocking) != cudaSuccess) ||
        (!ctx->evFork && cudaEventCreateWithFlags(&ctx->evFork, cudaEventDisableTiming) != cudaSuccess) ||
        (!ctx->evJoin && cudaEventCreateWithFlags(&ctx->evJoin, cudaEventDisableTiming) != cudaSuccess))
        return fail(ctx, IX_ERR_CUDA, "cudaStreamCreate failed");
    const int n = ctx->n;
    IX_TRY(deviceAlloc(ctx, "pos", 3 * (size_t)n, &ctx->dPos));
    // flags, term energies and interaction counts side by side, so that one copy brings them to the host
    unsigned char* status = nullptr;
    IX_TRY(deviceAlloc(ctx, "status", kStatusBytes, &status));
    ctx->dFlags = reinterpret_cast<int*>(status);
    ctx->dOutEnergy = reinterpret_cast<double*>(status + 32);
    ctx->dCounts = reinterpret_cast<unsigned long long*>(status + 64);
    IX_TRY(deviceAlloc(ctx, "outForces", 3 * (size_t)n, &ctx->dOutForces));
    IX_TRY(deviceAlloc(ctx, "energyBlocks", 4 * kReduceBlocks, &ctx->dEnergyBlocks));
    IX_TRY(deviceAlloc(ctx, "reduceTicket", 1, &ctx->dReduceTicket));
    int init[8] = {1, 0, 0, 0, 1, 0, 0, 0};
    IX_TRY(stageCopy(ctx, ctx->dFlags, init, sizeof(init)));
    IX_CUDA(ctx, cudaMemsetAsync(ctx->dReduceTicket, 0, sizeof(unsigned), ctx->stream));
    IX_CUDA(ctx, cudaMemsetAsync(ctx->dCounts, 0, 4 * sizeof(unsigned long long), ctx->stream));
    IX_TRY(uploadsDone(ctx));
    return IX_OK;
}

extern "C" {

const char* ix_version(void) { return "interax-b200 0.1 (sm_100a)"; }

int ix_measure_fp32_peak(int device, double* tflops) {
    if (!tflops) return fail(nullptr, IX_ERR_INVALID, "ix_measure_fp32_peak: tflops is NULL");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_NO_DEVICE, "cudaSetDevice(%d) failed: %s", device, cudaGetErrorString(e));
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    int perSM = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kFmaPeak, 256, 0);
    const int blocks = prop.multiProcessorCount * std::max(1, perSM);
    float* sink = nullptr;
    if (cudaMalloc(&sink, 256 * sizeof(float)) != cudaSuccess) return fail(nullptr, IX_ERR_CUDA, "cudaMalloc failed");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best = 0.0;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(a);
        kFmaPeak<<<blocks, 256>>>(sink, 1.0f + rep);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        double flops = 2.0 * (double)blocks * 256 * kProbeIters * kProbeChains;
        if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_CUDA, "FMA probe failed: %s", cudaGetErrorString(e));
    *tflops = best;
    return IX_OK;
}

int ix_ctx_create(int num_particles, int device, const double* default_box, ix_ctx** out) {
    if (!out) return fail(nullptr, IX_ERR_INVALID, "ix_ctx_create: out is NULL");
    *out = nullptr;
    if (num_particles <= 0) return fail(nullptr, IX_ERR_INVALID, "ix_ctx_create: the System has no particles");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(nullptr, IX_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= count)
        return fail(nullptr, IX_ERR_NO_DEVICE, "CUDA device %d does not exist (%d devices)", device, count);
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_CUDA, "cudaSetDevice(%d) failed: %s", device, cudaGetErrorString(e));
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    if (prop.major < 10)
        return fail(nullptr, IX_ERR_NO_DEVICE, "device %d (%s, sm_%d%d) is not a Blackwell (sm_100) GPU", device,
                    prop.name, prop.major, prop.minor);
    ix_ctx* ctx = new ix_ctx();
    ctx->n = num_particles;
    ctx->device = device;
    if (default_box) {
        std::memcpy(ctx->defaultBox, default_box, sizeof(ctx->defaultBox));
        std::memcpy(ctx->box, default_box, sizeof(ctx->box));
    }
    const int rc = ctxInitDevice(ctx);
    if (rc != IX_OK) {
        g_createError = ctx->error;
        ix_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return IX_OK;
}

void ix_ctx_destroy(ix_ctx* ctx) {
    if (!ctx) return;
    // a request described on the host only (device -1) has no device side: selecting device -1 would leave an
    // "invalid device" error for the next cudaGetLastError of whatever runs on this thread
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    releaseGraph(ctx->graphCompute);
    releaseGraph(ctx->graphDevice);
    releaseGraph(ctx->graphMd);
    releaseGraph(ctx->graphPosq);
    for (auto& g : ctx->graphWindows) releaseGraph(g);
    for (auto& kv : ctx->buffers) arenaFree(ctx->arena, kv.second.p);
    if (ctx->hostStatus) pinnedSlots().give(ctx->hostStatus);
    if (ctx->deviceStatus) pinnedSlots().give(ctx->deviceStatus);
    if (ctx->evStatus) cudaEventDestroy(ctx->evStatus);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->evFork) cudaEventDestroy(ctx->evFork);
    if (ctx->evJoin) cudaEventDestroy(ctx->evJoin);
    if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
    if (ctx->streamBody) cudaStreamDestroy(ctx->streamBody);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* ix_last_error(const ix_ctx* ctx) { return ctx ? ctx->error.c_str() : g_createError.c_str(); }

int ix_add_dispersion(ix_ctx* ctx, const ix_pair_settings* settings, const double* params, const uint8_t* alch,
                      double damping_scale, int use_lrc) {
    IX_TRY(addPairForce(ctx, 0, settings, params, alch, 5));
    ctx->term[0].dampingScale = damping_scale;
    ctx->term[0].useLrc = use_lrc != 0;
    return IX_OK;
}

int ix_add_exchange(ix_ctx* ctx, const ix_pair_settings* settings, const double* params, const uint8_t* alch,
                    int overlap_method) {
    if (ctx && overlap_method != 0 && overlap_method != 2)
        return fail(ctx, IX_ERR_INVALID, "InteraxExchangeForce: Illegal value for overlap method");
    IX_TRY(addPairForce(ctx, 1, settings, params, alch, 2));
    ctx->term[1].overlapMethod = overlap_method;
    return IX_OK;
}

int ix_add_short_range(ix_ctx* ctx, const ix_pair_settings* settings, const double* params, const uint8_t* alch,
                       int overlap_method) {
    if (ctx && overlap_method != 0 && overlap_method != 2)
        return fail(ctx, IX_ERR_INVALID, "InteraxShortRangeForce: Illegal value for overlap method");
    IX_TRY(addPairForce(ctx, 2, settings, params, alch, 3));
    ctx->term[2].overlapMethod = overlap_method;
    return IX_OK;
}

int ix_add_three_body(ix_ctx* ctx, int num_sites, const int32_t* site_offsets, const int32_t* site_particles,
                      const double* site_params, const int32_t* molecule, const uint8_t* alch, double cutoff,
                      double scale_factor, int damping_method, double damping_scale, double centroid_radius,
                      int periodic, const char* alch_name, int force_group) {
    if (!ctx) return IX_ERR_INVALID;
    if (ctx->atmPresent) return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: the context already has this force");
    if (num_sites < 0 || (num_sites > 0 && (!site_offsets || !site_particles || !site_params || !molecule || !alch)))
        return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: null argument");
    if (damping_method != IX_NO_DAMPING && damping_method != IX_TANG_TOENNIES)
        return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: Illegal value for damping method");
    if (centroid_radius < 0)
        return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: The centroid damping radius cannot be negative");
    // InteraxThreeBodyForceImpl::initialize (InteraxThreeBodyForceImpl.cpp:42-59)
    for (int s = 0; s < num_sites; s++) {
        if (site_offsets[s + 1] <= site_offsets[s])
            return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: A site must contain at least one particle");
        for (int k = site_offsets[s]; k < site_offsets[s + 1]; k++)
            if (site_particles[k] < 0 || site_particles[k] >= ctx->n)
                return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: Illegal particle index for a site");
        if (damping_method == IX_TANG_TOENNIES && site_params[3 * s + 2] <= 0)
            return fail(ctx, IX_ERR_INVALID,
                        "InteraxThreeBodyForce: The Tang-Toennies damping requires a positive width for every site");
    }
    if (cutoff <= 0) return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: The cutoff distance must be positive");
    if (force_group < 0 || force_group > 31)
        return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: Force group must be between 0 and 31");
    ctx->atmPresent = num_sites > 0;
    ctx->atmGroup = force_group;
    ctx->atmAlchName = alch_name ? alch_name : "lambda_sterics";
    ctx->siteOffsets.assign(site_offsets, site_offsets + num_sites + 1);
    ctx->siteParticles.assign(site_particles, site_particles + site_offsets[num_sites]);
    ctx->siteParams.assign(site_params, site_params + 3 * (size_t)num_sites);
    ctx->molecule.assign(molecule, molecule + num_sites);
    ctx->siteAlch.assign(alch, alch + num_sites);
    ctx->atmAnyAlch = std::any_of(ctx->siteAlch.begin(), ctx->siteAlch.end(), [](unsigned char a) { return a != 0; });
    ctx->atmCutoff = cutoff;
    ctx->atmScale = scale_factor;
    ctx->atmDamping = damping_method;
    ctx->atmDampingScale = damping_scale;
    ctx->atmCentroidRadius = centroid_radius;
    ctx->atmPeriodic = periodic != 0;
    ctx->atmAllocated = false;
    ctx->atmDirty = true;
    bumpVersion(ctx);
    return IX_OK;
}

static int updatePair(ix_ctx* ctx, int t, const double* params, int stride) {
    if (!ctx) return IX_ERR_INVALID;
    ctx->mdForcesValid = false;
    if (!ctx->term[t].present) return fail(ctx, IX_ERR_STATE, "%s: the context has no such force", kTermNames[t]);
    if (!params) return fail(ctx, IX_ERR_INVALID, "%s: null argument", kTermNames[t]);
    ctx->term[t].params.assign(params, params + (size_t)ctx->n * stride);
    ctx->pairDirty = true;
    ctx->pairShareOverlap = -1;
    bumpVersion(ctx);
    return IX_OK;
}

int ix_update_dispersion(ix_ctx* ctx, const double* params, double damping_scale) {
    IX_TRY(updatePair(ctx, 0, params, 5));
    ctx->term[0].dampingScale = damping_scale;
    return IX_OK;
}

int ix_update_exchange(ix_ctx* ctx, const double* params, int overlap_method) {
    if (ctx && ctx->term[1].present && overlap_method != ctx->term[1].overlapMethod)
        return fail(ctx, IX_ERR_INVALID, "updateParametersInContext: The overlap method has changed");
    return updatePair(ctx, 1, params, 2);
}

int ix_update_short_range(ix_ctx* ctx, const double* params, int overlap_method) {
    if (ctx && ctx->term[2].present && overlap_method != ctx->term[2].overlapMethod)
        return fail(ctx, IX_ERR_INVALID, "updateParametersInContext: The overlap method has changed");
    return updatePair(ctx, 2, params, 3);
}

int ix_update_three_body(ix_ctx* ctx, const double* site_params, double scale_factor, double damping_scale,
                         double centroid_radius) {
    if (!ctx) return IX_ERR_INVALID;
    ctx->mdForcesValid = false;
    if (!ctx->atmPresent) return fail(ctx, IX_ERR_STATE, "InteraxThreeBodyForce: the context has no such force");
    // the centroid damping cannot be switched on or off (CommonInteraxKernels.cpp:621-623)
    if ((centroid_radius > 0) != (ctx->atmCentroidRadius > 0))
        return fail(ctx, IX_ERR_INVALID,
                    "updateParametersInContext: The centroid damping cannot be switched on or off");
    if (centroid_radius < 0)
        return fail(ctx, IX_ERR_INVALID, "InteraxThreeBodyForce: The centroid damping radius cannot be negative");
    const int ns = (int)ctx->siteParams.size() / 3;
    if (ctx->atmDamping == IX_TANG_TOENNIES)
        for (int s = 0; s < ns; s++)
            if (site_params[3 * s + 2] <= 0)
                return fail(ctx, IX_ERR_INVALID,
                            "InteraxThreeBodyForce: The Tang-Toennies damping requires a positive width for every site");
    ctx->siteParams.assign(site_params, site_params + 3 * (size_t)ns);
    ctx->atmScale = scale_factor;
    ctx->atmDampingScale = damping_scale;
    ctx->atmCentroidRadius = centroid_radius;
    ctx->atmDirty = true;
    bumpVersion(ctx);
    return IX_OK;
}

int ix_dispersion_long_range_correction(int num_particles, const double* params, const uint8_t* is_alchemical,
                                        const ix_pair_settings* settings, double damping_scale,
                                        int use_long_range_correction, double* coefficient,
                                        double* alchemical_coefficient) {
    if (!coefficient || !alchemical_coefficient || !settings || num_particles < 0 ||
        (num_particles > 0 && (!params || !is_alchemical)))
        return fail(nullptr, IX_ERR_INVALID, "ix_dispersion_long_range_correction: invalid argument");
    *coefficient = *alchemical_coefficient = 0.0;
    if (settings->nonbonded_method != IX_CUTOFF_PERIODIC || !use_long_range_correction) return IX_OK;
    ixhost::longRangeCorrection(num_particles, params, is_alchemical, settings->cutoff,
                                settings->use_switching_function != 0, settings->switching_distance, damping_scale,
                                *coefficient, *alchemical_coefficient);
    return IX_OK;
}

int ix_set_parameter(ix_ctx* ctx, const char* name, double value) {
    if (!ctx || !name) return IX_ERR_INVALID;
    ctx->mdForcesValid = false;
    ctx->parameters[name] = value;
    bumpVersion(ctx);
    return IX_OK;
}

int ix_set_positions(ix_ctx* ctx, const double* positions, const double* box) {
    NvtxRange nvtxRange("ix_set_positions");
    if (!ctx) return IX_ERR_INVALID;
    ctx->mdForcesValid = false;
    if (!positions) return fail(ctx, IX_ERR_INVALID, "ix_set_positions: positions is NULL");
    for (size_t i = 0; i < 3 * (size_t)ctx->n; i++)
        if (!std::isfinite(positions[i]))
            return fail(ctx, IX_ERR_INVALID, "Particle coordinate is NaN or infinite (particle %zu)", i / 3);
    if (box) {
        if (box[0] <= 0 || box[4] <= 0 || box[8] <= 0)
            return fail(ctx, IX_ERR_INVALID, "Illegal periodic box vectors");
        if (std::memcmp(ctx->box, box, sizeof(ctx->box)) != 0) bumpVersion(ctx);
        std::memcpy(ctx->box, box, sizeof(ctx->box));
    }
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    IX_TRY(stageCopy(ctx, ctx->dPos, positions, 3 * (size_t)ctx->n * sizeof(double)));
    ctx->havePositions = true;
    ctx->mdPending.clear();
    return IX_OK;
}

// Enqueue one evaluation of the selected terms into dOutForces / dOutEnergy through the graph g, captured with the
// given key parameter.
static int enqueueResident(ix_ctx* ctx, unsigned terms, LaunchGraph& g, double param) {
    IX_TRY(stageUploads(ctx, terms));
    GraphKey key;
    key.terms = terms;
    key.out0 = ctx->dOutForces;
    key.out1 = ctx->dOutEnergy;
    key.param = param;
    return launchGraph(ctx, g, key, [&]() {
        return launchEvaluation(ctx, terms, ctx->dOutForces, ctx->dOutEnergy, nullptr, 0);
    });
}

// Record the interacting pair and triple counts of the last evaluation (synchronous).
static int readCounts(ix_ctx* ctx, unsigned terms) {
    unsigned long long c[2];
    IX_CUDA(ctx, cudaMemcpy(c, ctx->dCounts + 2, sizeof(c), cudaMemcpyDeviceToHost));
    ctx->lastPairs = (terms & 7u) ? (long long)c[0] : 0;
    ctx->lastTriples = (terms & 8u) ? (long long)c[1] : 0;
    return IX_OK;
}

// One evaluation of the selected terms at the current positions and parameters, left on the device: forces in
// dOutForces, term energies copied to e.  Grows the neighbor lists and repeats on an overflow.
static int evaluateResident(ix_ctx* ctx, unsigned terms, double e[4], LaunchGraph* graph = nullptr,
                            double param = 0.0, double* hostForces = nullptr) {
    for (int t = 0; t < 4; t++) e[t] = 0.0;
    if (!terms) return IX_OK;
    IX_TRY(prepare(ctx, terms));
    if (!ctx->hostStatus) ctx->hostStatus = pinnedSlots().take();
    unsigned char* hs = ctx->hostStatus;
    for (int attempt = 0; attempt < 4; attempt++) {
        IX_TRY(enqueueResident(ctx, terms, graph ? *graph : ctx->graphCompute, param));
        // the status block and the forces come back with the evaluation; one wait for all of it
        if (hs)
            IX_CUDA(ctx, cudaMemcpyAsync(hs, ctx->dFlags, kStatusBytes, cudaMemcpyDeviceToHost, ctx->stream));
        if (hostForces)
            IX_CUDA(ctx, cudaMemcpyAsync(hostForces, ctx->dOutForces, 3 * (size_t)ctx->n * sizeof(double),
                                         cudaMemcpyDeviceToHost, ctx->stream));
        IX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        bool redo = false;
        if (hs) IX_TRY(checkOverflowFlags(ctx, terms, reinterpret_cast<const int*>(hs), redo));
        else IX_TRY(checkOverflow(ctx, terms, redo));
        if (!redo) break;
    }
    unsigned long long c[2];
    if (hs) {
        std::memcpy(e, hs + 32, 4 * sizeof(double));
        std::memcpy(c, hs + 64 + 2 * sizeof(unsigned long long), sizeof(c));
    }
    else {
        IX_CUDA(ctx, cudaMemcpy(e, ctx->dOutEnergy, 4 * sizeof(double), cudaMemcpyDeviceToHost));
        IX_CUDA(ctx, cudaMemcpy(c, ctx->dCounts + 2, sizeof(c), cudaMemcpyDeviceToHost));
    }
    ctx->lastPairs = (terms & 7u) ? (long long)c[0] : 0;
    ctx->lastTriples = (terms & 8u) ? (long long)c[1] : 0;
    for (int t = 0; t < 4; t++)
        if (!((terms >> t) & 1u)) e[t] = 0.0;
    return IX_OK;
}

int ix_compute(ix_ctx* ctx, int groups, int include_forces, int include_energy, double* term_energies,
               double* energy, double* forces) {
    NvtxRange nvtxRange("ix_compute");
    if (!ctx) return IX_ERR_INVALID;
    ctx->mdForcesValid = false;
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned terms = selectedTerms(ctx, groups);
    double e[4];
    const bool copyForces = forces && terms && include_forces;
    IX_TRY(evaluateResident(ctx, terms, e, nullptr, 0.0, copyForces ? forces : nullptr));
    if (term_energies) std::memcpy(term_energies, e, sizeof(e));
    if (energy) *energy = e[0] + e[1] + e[2] + e[3];
    if (forces && !copyForces) std::memset(forces, 0, 3 * (size_t)ctx->n * sizeof(double));
    (void)include_energy;
    return IX_OK;
}

}  // extern "C"

// The device entry points do not wait for their work.  Each records its flags (list overflows) into pinned memory
// with an event after them; the next device call, or ix_get_device_status, waits for that event and grows the lists
// that overflowed, so that a call repeated after an overflow is complete (as OpenMM repeats a force evaluation whose
// neighbor list overflowed).
static int deviceStatusCheck(ix_ctx* ctx) {
    if (!ctx->statusPending) return IX_OK;
    IX_CUDA(ctx, cudaEventSynchronize(ctx->evStatus));
    ctx->statusPending = false;
    const int* flags = reinterpret_cast<const int*>(ctx->deviceStatus);
    ctx->lastDeviceStatus = (flags[1] ? 1 : 0) | (flags[5] ? 2 : 0);
    if (ctx->lastDeviceStatus) {
        bool redo = false;
        IX_TRY(checkOverflowFlags(ctx, selectedTerms(ctx, -1), flags, redo));
    }
    return IX_OK;
}

__global__ void kDeviceStatus(const int* flags, const double* termEnergies, unsigned terms, double* addEnergy,
                              int* status) {
    if (status) *status = (flags[1] ? 1 : 0) | (flags[5] ? 2 : 0);
    if (addEnergy) {
        double e = 0.0;
        for (int t = 0; t < 4; t++)
            if ((terms >> t) & 1u) e += termEnergies[t];
        *addEnergy += e;
    }
}

static int deviceStatusRecord(ix_ctx* ctx) {
    if (!ctx->deviceStatus) ctx->deviceStatus = pinnedSlots().take();
    if (!ctx->evStatus) IX_CUDA(ctx, cudaEventCreateWithFlags(&ctx->evStatus, cudaEventDisableTiming));
    if (!ctx->deviceStatus) return fail(ctx, IX_ERR_CUDA, "pinned host memory for the status is not available");
    IX_CUDA(ctx, cudaMemcpyAsync(ctx->deviceStatus, ctx->dFlags, 8 * sizeof(int), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    IX_CUDA(ctx, cudaEventRecord(ctx->evStatus, ctx->stream));
    ctx->statusPending = true;
    return IX_OK;
}

// Positions of a caller's device array in its slot order (slot k holds particle atomIndex[k], or k) into the
// context's FP64 positions, and the slot of each particle for the force rows.  FORMAT: IX_POSQ_FLOAT4,
// IX_POSQ_FLOAT4_CORRECTED (x = posq.x + correction.x, OpenMM's mixed precision), IX_POSQ_DOUBLE4.
template <int FORMAT>
__global__ void kGatherPosq(int n, const void* posq, const float4* correction, const int* atomIndex, double* pos,
                            int* slotOfParticle) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = atomIndex ? atomIndex[k] : k;
    if (i < 0 || i >= n) return;
    double x, y, z;
    if (FORMAT == IX_POSQ_DOUBLE4) {
        const double4 p = reinterpret_cast<const double4*>(posq)[k];
        x = p.x;
        y = p.y;
        z = p.z;
    }
    else {
        const float4 p = reinterpret_cast<const float4*>(posq)[k];
        x = p.x;
        y = p.y;
        z = p.z;
        if (FORMAT == IX_POSQ_FLOAT4_CORRECTED) {
            const float4 c = correction[k];
            x += c.x;
            y += c.y;
            z += c.z;
        }
    }
    pos[3 * i] = x;
    pos[3 * i + 1] = y;
    pos[3 * i + 2] = z;
    slotOfParticle[i] = k;
}

extern "C" {

int ix_set_list_capacity(ix_ctx* ctx, long long pair_tiles, int site_neighbors) {
    if (!ctx) return IX_ERR_INVALID;
    if (pair_tiles < 0 || site_neighbors < 0) return fail(ctx, IX_ERR_INVALID, "ix_set_list_capacity: negative capacity");
    ctx->tileCapRequest = pair_tiles;
    ctx->atmCap = site_neighbors;
    ctx->pairAllocated = false;
    ctx->atmAllocated = false;
    bumpVersion(ctx);
    return IX_OK;
}

int ix_get_list_stats(ix_ctx* ctx, long long* pair_tiles, int* site_neighbors, long long* md_reruns) {
    if (!ctx) return IX_ERR_INVALID;
    if (pair_tiles) *pair_tiles = ctx->pairAllocated ? ctx->tileCap : 0;
    if (site_neighbors) *site_neighbors = ctx->atmAllocated ? ctx->atmCap : 0;
    if (md_reruns) *md_reruns = ctx->mdReruns;
    return IX_OK;
}

int ix_get_device_status(ix_ctx* ctx, int* status) {
    if (!ctx || !status) return IX_ERR_INVALID;
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    IX_TRY(deviceStatusCheck(ctx));
    *status = ctx->lastDeviceStatus;
    return IX_OK;
}

int ix_compute_device_posq(ix_ctx* ctx, int groups, int posq_format, const void* d_posq,
                           const void* d_posq_correction, const int32_t* d_atom_index, const double* box,
                           long long* d_force_fixed, int force_stride, double* d_energy, int* d_status) {
    NvtxRange nvtxRange("ix_compute_device_posq");
    if (!ctx) return IX_ERR_INVALID;
    if (posq_format != IX_POSQ_FLOAT4 && posq_format != IX_POSQ_FLOAT4_CORRECTED && posq_format != IX_POSQ_DOUBLE4)
        return fail(ctx, IX_ERR_INVALID, "ix_compute_device_posq: unknown position format %d", posq_format);
    if (!d_posq || (posq_format == IX_POSQ_FLOAT4_CORRECTED && !d_posq_correction))
        return fail(ctx, IX_ERR_INVALID, "ix_compute_device_posq: positions are NULL");
    if (d_force_fixed && force_stride < ctx->n)
        return fail(ctx, IX_ERR_INVALID, "ix_compute_device_posq: stride smaller than the particle count");
    ctx->mdForcesValid = false;
    ctx->mdPending.clear();
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    IX_TRY(deviceStatusCheck(ctx));
    if (box) {
        if (box[0] <= 0 || box[4] <= 0 || box[8] <= 0) return fail(ctx, IX_ERR_INVALID, "Illegal periodic box vectors");
        if (std::memcmp(ctx->box, box, sizeof(ctx->box)) != 0) bumpVersion(ctx);
        std::memcpy(ctx->box, box, sizeof(ctx->box));
    }
    ctx->havePositions = true;
    unsigned terms = selectedTerms(ctx, groups);
    if (!ctx->dAddSlot) {
        IX_TRY(deviceAlloc(ctx, "addSlot", ctx->n, &ctx->dAddSlot));
        IX_CUDA(ctx, cudaMemsetAsync(ctx->dAddSlot, 0xff, ctx->n * sizeof(int), ctx->stream));   // -1: no slot yet
    }
    if (terms) {
        IX_TRY(prepare(ctx, terms));
        IX_TRY(stageUploads(ctx, terms));
    }
    GraphKey key;
    key.terms = terms;
    key.out0 = d_energy;
    key.out2 = d_force_fixed;
    key.out3 = d_status;
    key.in0 = d_posq;
    key.in1 = d_posq_correction;
    key.in2 = d_atom_index;
    key.format = posq_format;
    key.stride = force_stride;
    IX_TRY(launchGraph(ctx, ctx->graphPosq, key, [&]() -> int {
        const int blocks = (ctx->n + 255) / 256;
        const float4* corr = reinterpret_cast<const float4*>(d_posq_correction);
        if (posq_format == IX_POSQ_DOUBLE4)
            kGatherPosq<IX_POSQ_DOUBLE4><<<blocks, 256, 0, ctx->stream>>>(ctx->n, d_posq, corr, d_atom_index,
                                                                           ctx->dPos, ctx->dAddSlot);
        else if (posq_format == IX_POSQ_FLOAT4_CORRECTED)
            kGatherPosq<IX_POSQ_FLOAT4_CORRECTED><<<blocks, 256, 0, ctx->stream>>>(ctx->n, d_posq, corr, d_atom_index,
                                                                                    ctx->dPos, ctx->dAddSlot);
        else
            kGatherPosq<IX_POSQ_FLOAT4><<<blocks, 256, 0, ctx->stream>>>(ctx->n, d_posq, corr, d_atom_index,
                                                                          ctx->dPos, ctx->dAddSlot);
        ctx->launches += 1;
        if (terms)
            IX_TRY(launchEvaluation(ctx, terms, nullptr, ctx->dOutEnergy, d_force_fixed, force_stride, nullptr,
                                    ctx->dAddSlot));
        kDeviceStatus<<<1, 1, 0, ctx->stream>>>(ctx->dFlags, ctx->dOutEnergy, terms, d_energy, d_status);
        ctx->launches += 1;
        IX_CUDA(ctx, cudaGetLastError());
        return IX_OK;
    }));
    return deviceStatusRecord(ctx);
}

int ix_compute_device(ix_ctx* ctx, int groups, long long* d_force_fixed, int force_stride, double* d_term_energies) {
    NvtxRange nvtxRange("ix_compute_device");
    if (!ctx) return IX_ERR_INVALID;
    if (force_stride < ctx->n) return fail(ctx, IX_ERR_INVALID, "ix_compute_device: stride smaller than the particle count");
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    IX_TRY(deviceStatusCheck(ctx));
    unsigned terms = selectedTerms(ctx, groups);
    if (!terms) return IX_OK;
    IX_TRY(prepare(ctx, terms));
    IX_TRY(stageUploads(ctx, terms));
    GraphKey key;
    key.terms = terms;
    key.out1 = d_term_energies;
    key.out2 = d_force_fixed;
    key.stride = force_stride;
    IX_TRY(launchGraph(ctx, ctx->graphDevice, key, [&]() {
        return launchEvaluation(ctx, terms, nullptr, d_term_energies, d_force_fixed, force_stride);
    }));
    return deviceStatusRecord(ctx);
}

int ix_compute_device_f64(ix_ctx* ctx, int groups, const double* d_positions, const double* box, double* d_forces,
                          double* d_term_energies) {
    NvtxRange nvtxRange("ix_compute_device_f64");
    if (!ctx) return IX_ERR_INVALID;
    ctx->mdForcesValid = false;
    ctx->mdPending.clear();
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    IX_TRY(deviceStatusCheck(ctx));
    if (box) {
        if (box[0] <= 0 || box[4] <= 0 || box[8] <= 0) return fail(ctx, IX_ERR_INVALID, "Illegal periodic box vectors");
        if (std::memcmp(ctx->box, box, sizeof(ctx->box)) != 0) bumpVersion(ctx);
        std::memcpy(ctx->box, box, sizeof(ctx->box));
    }
    if (d_positions) {
        IX_CUDA(ctx, cudaMemcpyAsync(ctx->dPos, d_positions, 3 * (size_t)ctx->n * sizeof(double),
                                     cudaMemcpyDeviceToDevice, ctx->stream));
        ctx->havePositions = true;
    }
    unsigned terms = selectedTerms(ctx, groups);
    if (!terms) {
        if (d_forces) IX_CUDA(ctx, cudaMemsetAsync(d_forces, 0, 3 * (size_t)ctx->n * sizeof(double), ctx->stream));
        if (d_term_energies) IX_CUDA(ctx, cudaMemsetAsync(d_term_energies, 0, 4 * sizeof(double), ctx->stream));
        return IX_OK;
    }
    IX_TRY(prepare(ctx, terms));
    IX_TRY(stageUploads(ctx, terms));
    GraphKey key;
    key.terms = terms;
    key.out0 = d_forces;
    key.out1 = d_term_energies;
    IX_TRY(launchGraph(ctx, ctx->graphDevice, key,
                       [&]() { return launchEvaluation(ctx, terms, d_forces, d_term_energies, nullptr, 0); }));
    return deviceStatusRecord(ctx);
}

int ix_set_counting(ix_ctx* ctx, int enable) {
    if (!ctx) return IX_ERR_INVALID;
    ctx->counting = enable != 0;
    bumpVersion(ctx);
    return IX_OK;
}

int ix_get_counts(ix_ctx* ctx, long long* num_pairs, long long* num_triples) {
    if (!ctx) return IX_ERR_INVALID;
    if (num_pairs) *num_pairs = ctx->lastPairs;
    if (num_triples) *num_triples = ctx->lastTriples;
    return IX_OK;
}

void* ix_get_stream(ix_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int ix_synchronize(ix_ctx* ctx) {
    if (!ctx) return IX_ERR_INVALID;
    IX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    IX_CUDA(ctx, cudaGetLastError());
    return IX_OK;
}

int ix_md_set_masses(ix_ctx* ctx, const double* masses) {
    if (!ctx || !masses) return IX_ERR_INVALID;
    std::vector<double> inv(ctx->n);
    for (int i = 0; i < ctx->n; i++) {
        if (!(masses[i] >= 0)) return fail(ctx, IX_ERR_INVALID, "Illegal mass for particle %d", i);
        inv[i] = masses[i] > 0 ? 1.0 / masses[i] : 0.0;
    }
    IX_TRY(deviceAlloc(ctx, "invMass", ctx->n, &ctx->dInvMass));
    IX_TRY(deviceAlloc(ctx, "vel", 3 * (size_t)ctx->n, &ctx->dVel));
    IX_TRY(stageCopy(ctx, ctx->dInvMass, inv.data(), ctx->n * sizeof(double)));
    ctx->haveMasses = true;
    ctx->mdPending.clear();
    bumpVersion(ctx);
    return IX_OK;
}

int ix_set_profiling(ix_ctx* ctx, int enable) {
    if (!ctx) return IX_ERR_INVALID;
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    if (enable && !ctx->ev[0])
        for (auto& e : ctx->ev) IX_CUDA(ctx, cudaEventCreate(&e));
    ctx->profiling = enable != 0;
    ctx->serialize = enable == 2;
    bumpVersion(ctx);
    ctx->evPair = ctx->evAtm = false;
    return IX_OK;
}

int ix_get_kernel_times(ix_ctx* ctx, double* pair_ms, double* three_body_ms) {
    if (!ctx) return IX_ERR_INVALID;
    float ms = 0.0f;
    if (pair_ms) {
        *pair_ms = 0.0;
        if (ctx->evPair) {
            IX_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
            IX_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
            *pair_ms = ms;
        }
    }
    if (three_body_ms) {
        *three_body_ms = 0.0;
        if (ctx->evAtm) {
            IX_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
            IX_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
            *three_body_ms = ms;
        }
    }
    return IX_OK;
}

}  // extern "C"

// Enqueue velocity-Verlet steps on the context's stream without synchronizing.
static int enqueueSteps(ix_ctx* ctx, int num_steps, double dt) {
    unsigned terms = selectedTerms(ctx, -1);
    if (terms) {
        IX_TRY(prepare(ctx, terms));
        IX_TRY(stageUploads(ctx, terms));
    }
    const int n = ctx->n;
    const int g = (n + 255) / 256;
    if (!ctx->mdForcesValid) {
        if (terms) IX_TRY(launchEvaluation(ctx, terms, ctx->dOutForces, ctx->dOutEnergy, nullptr, 0));
        else IX_CUDA(ctx, cudaMemsetAsync(ctx->dOutForces, 0, 3 * (size_t)n * sizeof(double), ctx->stream));
        ctx->mdForcesValid = true;
    }
    // one step = half kick + drift, the evaluation at the new positions, half kick; replayed as one graph
    GraphKey key;
    key.terms = terms;
    key.out0 = ctx->dOutForces;
    key.out1 = ctx->dOutEnergy;
    key.dt = dt;
    // one step: the first half kick and drift (fused with the list's displacement check and position refresh when
    // there are pair terms), the evaluation at the new positions, whose finishing kernel applies the second half kick
    const int clusterGrid = (ctx->K.num + kClusterBlock - 1) / kClusterBlock;
    auto step = [&]() -> int {
        if (!terms) {
            if (ctx->numConstraints)
                kConstrainedDrift<<<clusterGrid, kClusterBlock, 0, ctx->stream>>>(
                    ctx->K, dt, ctx->dInvMass, ctx->dOutForces, ctx->dVel, ctx->dPos, ctx->L, false, 0.0f);
            else
                kVerletFirstHalf<<<g, 256, 0, ctx->stream>>>(n, dt, ctx->dInvMass, ctx->dOutForces, ctx->dVel,
                                                             ctx->dPos);
            kVerletSecondHalf<<<g, 256, 0, ctx->stream>>>(n, dt, ctx->dInvMass, ctx->dOutForces, ctx->dVel);
            ctx->launches += 2;
            if (ctx->numConstraints) {
                kConstrainVelocities<<<clusterGrid, kClusterBlock, 0, ctx->stream>>>(ctx->K, ctx->dInvMass,
                                                                                    ctx->dPos, ctx->dVel);
                ctx->launches += 1;
            }
            IX_CUDA(ctx, cudaGetLastError());
            return IX_OK;
        }
        StepKick kick{ctx->dInvMass, ctx->dVel, 0.5 * dt};
        if (ctx->numConstraints) {
            // the constrained clusters move together, and refresh the pair list's sorted positions with the
            // displacement check as kStepStart does
            kConstrainedDrift<<<clusterGrid, kClusterBlock, 0, ctx->stream>>>(
                ctx->K, dt, ctx->dInvMass, ctx->dOutForces, ctx->dVel, ctx->dPos, ctx->L, (terms & 7u) != 0,
                0.25f * kPairSkin * kPairSkin);
        }
        else if (terms & 7u)
            // 128-thread blocks: a latency-bound gather by particle, spread over every SM
            kStepStart<<<(n + 127) / 128, 128, 0, ctx->stream>>>(ctx->L, ctx->dPos, dt, ctx->dInvMass, ctx->dOutForces,
                                                                ctx->dVel, 0.25f * kPairSkin * kPairSkin);
        else
            kVerletFirstHalf<<<g, 256, 0, ctx->stream>>>(n, dt, ctx->dInvMass, ctx->dOutForces, ctx->dVel, ctx->dPos);
        ctx->launches += 1;
        IX_TRY(launchEvaluation(ctx, terms, ctx->dOutForces, ctx->dOutEnergy, nullptr, 0, &kick));
        if (ctx->numConstraints) {
            kConstrainVelocities<<<clusterGrid, kClusterBlock, 0, ctx->stream>>>(ctx->K, ctx->dInvMass, ctx->dPos,
                                                                                ctx->dVel);
            ctx->launches += 1;
        }
        IX_CUDA(ctx, cudaGetLastError());
        return IX_OK;
    };
    for (int s = 0; s < num_steps; s++) IX_TRY(launchGraph(ctx, ctx->graphMd, key, step));
    IX_CUDA(ctx, cudaGetLastError());
    return IX_OK;
}

// The MD state (positions, velocities, forces, energies) copied to or from the save area, in stream order.
static int mdStateCopy(ix_ctx* ctx, bool save) {
    const size_t n3 = 3 * (size_t)ctx->n;
    IX_TRY(deviceAlloc(ctx, "mdSave", 3 * n3 + 4, &ctx->dMdSave));
    double* live[4] = {ctx->dPos, ctx->dVel, ctx->dOutForces, ctx->dOutEnergy};
    const size_t count[4] = {n3, n3, n3, 4};
    size_t off = 0;
    for (int k = 0; k < 4; k++) {
        double* kept = ctx->dMdSave + off;
        IX_CUDA(ctx, cudaMemcpyAsync(save ? kept : live[k], save ? live[k] : kept, count[k] * sizeof(double),
                                     cudaMemcpyDeviceToDevice, ctx->stream));
        off += count[k];
    }
    return IX_OK;
}

extern "C" {

// Enqueue velocity-Verlet steps without synchronizing (masses and velocities must have been set by ix_md_run or
// ix_md_set_state).  The first call after a finish saves the state, so that ix_md_finish can rerun the steps after a
// neighbor-list overflow.
int ix_md_steps_async(ix_ctx* ctx, int num_steps, double dt) {
    NvtxRange nvtxRange("ix_md_steps_async");
    if (!ctx) return IX_ERR_INVALID;
    if (!ctx->haveMasses) return fail(ctx, IX_ERR_STATE, "ix_md_steps_async: masses have not been set");
    if (!ctx->havePositions) return fail(ctx, IX_ERR_STATE, "positions have not been set");
    if (num_steps < 0) return fail(ctx, IX_ERR_INVALID, "ix_md_steps_async: negative step count");
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    if (ctx->mdRollback && (selectedTerms(ctx, -1) & 7u)) {
        if (ctx->mdPending.empty()) {
            IX_TRY(mdStateCopy(ctx, true));
            ctx->mdSavedForcesValid = ctx->mdForcesValid;
        }
        ctx->mdPending.push_back({num_steps, dt});
    }
    return enqueueSteps(ctx, num_steps, dt);
}

int ix_set_graphs(ix_ctx* ctx, int enable) {
    if (!ctx) return IX_ERR_INVALID;
    ctx->useGraphs = enable != 0;
    bumpVersion(ctx);
    return IX_OK;
}

// out[w] = (accumulate ? out[w] : 0) + f0 + lambda_w (f1 - f0): the forces of terms linear in the window parameter at
// each window, FP64, n x 3 per window.
__global__ void kWindowForces(size_t n3, int num_windows, const double* __restrict__ lambdas,
                              const double* __restrict__ f0, const double* __restrict__ f1, double* __restrict__ out,
                              int accumulate) {
    for (int w = blockIdx.y; w < num_windows; w += gridDim.y) {
        const double lam = lambdas[w];
        double* o = out + (size_t)w * n3;
        for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += (size_t)gridDim.x * blockDim.x) {
            const double v = fma(lam, f1[k] - f0[k], f0[k]);
            o[k] = accumulate ? o[k] + v : v;
        }
    }
}

// out[w] += base + a0 + lambda_w (a1 - a0) (a0, a1 may be null): the λ-independent and linear parts of the windows'
// forces added to their alchemical-pair parts.
__global__ void kWindowCombine(size_t n3, int num_windows, const double* __restrict__ lambdas,
                               const double* __restrict__ base, const double* __restrict__ a0,
                               const double* __restrict__ a1, double* __restrict__ out) {
    for (int w = blockIdx.y; w < num_windows; w += gridDim.y) {
        const double lam = lambdas[w];
        double* o = out + (size_t)w * n3;
        for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += (size_t)gridDim.x * blockDim.x) {
            double v = base[k];
            if (a0) v += fma(lam, a1[k] - a0[k], a0[k]);
            o[k] += v;
        }
    }
}

// Tiles holding at least one particle that carries the alchemical flag `bit` (1 or 0 per tile).
__global__ void kMarkAlchemicalTiles(ListBuffers L, const int* flags, int bit, unsigned char* out) {
    const int numTiles = min(*L.numTiles, L.tileCap);
    const int lane = threadIdx.x & 31;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < numTiles; t += (gridDim.x * blockDim.x) >> 5) {
        const int si = L.tileIBlock[t] * 32 + lane, sj = L.tileJ[32 * t + lane];
        const bool a = (flags[si] & bit) != 0 || (sj >= 0 && (flags[sj] & bit) != 0);
        const bool any = __any_sync(0xffffffffu, a);
        if (lane == 0) out[t] = any ? 1 : 0;
    }
}

static const size_t kMaxWindowGraphs = 40;

// The graph of an evaluation of the given terms at one value of the window parameter: the cached one, a new slot, or
// (when the cache is full) the slot replaced longest ago.  The reference is used at once, before the cache grows.
static LaunchGraph& windowGraph(ix_ctx* ctx, unsigned terms, double value) {
    for (auto& g : ctx->graphWindows)
        if (g.exec && g.key.terms == terms && std::memcmp(&g.key.param, &value, sizeof(value)) == 0) return g;
    if (ctx->graphWindows.size() < kMaxWindowGraphs) {
        ctx->graphWindows.emplace_back();
        return ctx->graphWindows.back();
    }
    return ctx->graphWindows[ctx->windowNext++ % ctx->graphWindows.size()];
}

// One pass over the windows (see computeWindows).  redo: a neighbor list overflowed after the first window and was
// grown; the pass must be repeated.
// Soft-core windows when every pair term uses the window parameter with the same alchemical particles: the pair terms
// are evaluated once at 0, where the alchemical pairs contribute nothing (their scale is the parameter), the
// three-body term at 0 and 1 (it is linear), and each window adds only its alchemical pairs: the pair kernel over the
// tiles that hold an alchemical particle, keeping the pairs with exactly one (the same kernel and terms as a full
// evaluation at that value).  The long-range correction's alchemical part joins each window's energy.
static int softcoreWindows(ix_ctx* ctx, const std::string& name, int num_windows, const double* values,
                           double* energies, double* d_forces) {
    const size_t n3 = 3 * (size_t)ctx->n;
    const unsigned terms = selectedTerms(ctx, -1), pairTerms = terms & 7u;
    const bool atmLinear = (terms & 8u) && ctx->atmAnyAlch && ctx->atmAlchName == name;
    int bit = 0;
    for (int t = 0; t < 3 && !bit; t++)
        if ((pairTerms >> t) & 1u) bit = 1 << t;
    double *dBase = nullptr, *dA0 = nullptr, *dA1 = nullptr, *dLambda = nullptr, *dWinEnergy = nullptr;
    double* dAlchEnergy = nullptr;
    int* dAlchCount = nullptr;
    unsigned long long* dPairScratch = nullptr;
    IX_TRY(deviceAlloc(ctx, "windowLambda", (size_t)num_windows, &dLambda));
    IX_TRY(deviceAlloc(ctx, "windowEnergy", 4 * (size_t)num_windows, &dWinEnergy));
    IX_TRY(deviceAlloc(ctx, "windowAlchCount", 1, &dAlchCount));
    IX_TRY(deviceAlloc(ctx, "windowPairScratch", 1, &dPairScratch));
    if (d_forces) {
        IX_TRY(deviceAlloc(ctx, "windowBase", n3, &dBase));
        if (terms & 8u) IX_TRY(deviceAlloc(ctx, "windowA0", n3, &dA0));
        if (atmLinear) IX_TRY(deviceAlloc(ctx, "windowSlope", n3, &dA1));
    }
    // the pair terms at 0 (the lists are built for these positions here), the three-body term at 0 and 1
    double eP[4], eA0[4] = {0, 0, 0, 0}, eA1[4] = {0, 0, 0, 0};
    ctx->parameters[name] = 0.0;
    IX_TRY(evaluateResident(ctx, pairTerms, eP, &windowGraph(ctx, pairTerms, 0.0), 0.0));
    const long long pairs = ctx->lastPairs;
    if (d_forces)
        IX_CUDA(ctx, cudaMemcpyAsync(dBase, ctx->dOutForces, n3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    long long triples = 0;
    if (terms & 8u) {
        IX_TRY(evaluateResident(ctx, 8u, eA0, &windowGraph(ctx, 8u, 0.0), 0.0));
        triples = ctx->lastTriples;
        if (d_forces)
            IX_CUDA(ctx, cudaMemcpyAsync(dA0, ctx->dOutForces, n3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        if (atmLinear) {
            ctx->parameters[name] = 1.0;
            IX_TRY(evaluateResident(ctx, 8u, eA1, &windowGraph(ctx, 8u, 1.0), 1.0));
            if (d_forces)
                IX_CUDA(ctx, cudaMemcpyAsync(dA1, ctx->dOutForces, n3 * sizeof(double), cudaMemcpyDeviceToDevice,
                                             ctx->stream));
        }
        else std::memcpy(eA1, eA0, sizeof(eA0));
    }
    // the tiles that hold an alchemical particle, in tile order
    int numTiles = 0;
    IX_CUDA(ctx, cudaMemcpy(&numTiles, ctx->L.numTiles, sizeof(int), cudaMemcpyDeviceToHost));
    numTiles = std::min(numTiles, ctx->tileCap);
    unsigned char* dMarks = nullptr;
    IX_TRY(deviceAlloc(ctx, "windowTileMarks", std::max(numTiles, 1), &dMarks));
    kMarkAlchemicalTiles<<<ctx->numSMs * 8, 256, 0, ctx->stream>>>(ctx->L, ctx->P.flags, bit, dMarks);
    ctx->launches += 1;
    std::vector<unsigned char> marks(std::max(numTiles, 1));
    IX_CUDA(ctx, cudaMemcpyAsync(marks.data(), dMarks, numTiles, cudaMemcpyDeviceToHost, ctx->stream));
    IX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<int> tiles;
    for (int t = 0; t < numTiles; t++)
        if (marks[t]) tiles.push_back(t);
    const int numTasks = (int)tiles.size();
    int* dTiles = nullptr;
    IX_TRY(deviceAlloc(ctx, "windowTiles", std::max(numTasks, 1), &dTiles));
    IX_TRY(deviceAlloc(ctx, "windowAlchEnergy", 3 * (size_t)std::max(numTasks, 1), &dAlchEnergy));
    if (numTasks) IX_TRY(stageCopy(ctx, dTiles, tiles.data(), tiles.size() * sizeof(int)));
    IX_TRY(stageCopy(ctx, dAlchCount, &numTasks, sizeof(int)));
    // each window: its alchemical pairs, then their forces and energies
    const PairTerm& D = ctx->term[0];
    const double volume = ctx->box[0] * ctx->box[4] * ctx->box[8];
    const int n = ctx->n;
    for (int w = 0; w < num_windows; w++) {
        ctx->parameters[name] = values[w];
        PairTermConfig C = pairConfig(ctx, pairTerms);
        C.alchOnlyBit = bit;
        PairBuffers P = ctx->P;
        P.taskTiles = dTiles;
        P.numTasks = numTasks;
        P.taskEnergy = dAlchEnergy;
        P.pairCount = dPairScratch;
        const bool table = P.coef != nullptr && C.overlapMethod[1] == 0 && C.overlapMethod[2] == 0;
        if (numTasks) {
            if (table) kPairTiles<false, true><<<ctx->pairGridBlocks, 32 * kPairWarps, 0, ctx->stream>>>(ctx->L, P, C);
            else kPairTiles<false, false><<<ctx->pairGridBlocks, 32 * kPairWarps, 0, ctx->stream>>>(ctx->L, P, C);
        }
        FinishForces F{};
        F.n = n;
        F.np = ctx->L.np;
        F.slotOf = ctx->L.slotOf;
        F.pairForce = ctx->P.forceFixed;
        F.outForces = d_forces ? d_forces + (size_t)w * n3 : nullptr;
        F.blocks = (n + 255) / 256;
        const double lrc = (D.present && (pairTerms & 1u) && D.lrcAlchCoef != 0) ? values[w] * D.lrcAlchCoef / volume
                                                                                 : 0.0;
        EnergyReduction R{dAlchEnergy, dAlchCount, std::max(numTasks, 1), nullptr, 0, lrc, dWinEnergy + 4 * (size_t)w,
                          ctx->dEnergyBlocks, ctx->dReduceTicket, nullptr, ctx->L.taskCounter};
        kFinish<<<F.blocks + kReduceBlocks, 256, 0, ctx->stream>>>(F, R);
        ctx->launches += numTasks ? 2 : 1;
        IX_CUDA(ctx, cudaGetLastError());
    }
    std::vector<double> alch(4 * (size_t)num_windows);
    IX_CUDA(ctx, cudaMemcpyAsync(alch.data(), dWinEnergy, alch.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    if (d_forces) {
        IX_TRY(stageCopy(ctx, dLambda, values, num_windows * sizeof(double)));
        const unsigned bx = (unsigned)std::max<size_t>(std::min<size_t>((n3 + 255) / 256, 1184), 1);
        const dim3 grid(bx, (unsigned)std::min(num_windows, 65535));
        kWindowCombine<<<grid, 256, 0, ctx->stream>>>(n3, num_windows, dLambda, dBase, dA0, atmLinear ? dA1 : dA0,
                                                      d_forces);
        ctx->launches += 1;
        IX_CUDA(ctx, cudaGetLastError());
    }
    IX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int w = 0; w < num_windows; w++) {
        for (int k = 0; k < 3; k++) energies[4 * w + k] = eP[k] + alch[4 * (size_t)w + k];
        energies[4 * w + 3] = eA0[3] + values[w] * (eA1[3] - eA0[3]);
    }
    ctx->lastPairs = pairs;
    ctx->lastTriples = triples;
    return IX_OK;
}

static int windowsPass(ix_ctx* ctx, const std::string& name, int num_windows, const double* values, double* energies,
                       double* d_forces, bool& redo) {
    redo = false;
    const size_t n3 = 3 * (size_t)ctx->n;
    const unsigned terms = selectedTerms(ctx, -1);
    bool pairNonlinear = false;
    for (int t = 0; t < 3; t++) {
        const PairTerm& T = ctx->term[t];
        pairNonlinear = pairNonlinear || (T.present && T.anyAlch && T.alchName == name && T.softcoreRadius > 0);
    }
    const unsigned pairTerms = terms & 7u;
    if (pairNonlinear) {
        // every pair term on the window parameter with a soft core and the same alchemical particles: only the
        // alchemical pairs are evaluated per window
        bool same = true;
        const PairTerm* first = nullptr;
        for (int t = 0; t < 3 && same; t++) {
            const PairTerm& T = ctx->term[t];
            if (!((pairTerms >> t) & 1u)) continue;
            same = T.anyAlch && T.alchName == name && T.softcoreRadius > 0 && (!first || T.alch == first->alch);
            if (!first) first = &T;
        }
        if (same) return softcoreWindows(ctx, name, num_windows, values, energies, d_forces);
    }
    const unsigned linearTerms = pairNonlinear ? (terms & 8u) : terms;
    double *dLin0 = nullptr, *dLin1 = nullptr, *dLambda = nullptr, *dWinEnergy = nullptr;
    IX_TRY(deviceAlloc(ctx, "windowLambda", (size_t)num_windows, &dLambda));
    if (linearTerms && d_forces) IX_TRY(deviceAlloc(ctx, "windowBase", n3, &dLin0));
    if (linearTerms && d_forces && pairNonlinear) IX_TRY(deviceAlloc(ctx, "windowSlope", n3, &dLin1));
    if (pairNonlinear) IX_TRY(deviceAlloc(ctx, "windowEnergy", 4 * (size_t)num_windows, &dWinEnergy));
    // the terms linear in the parameter: evaluated at 0 and 1
    double e0[4] = {0, 0, 0, 0}, e1[4] = {0, 0, 0, 0};
    long long pairs = 0, triples = 0;
    if (linearTerms) {
        ctx->parameters[name] = 0.0;
        IX_TRY(evaluateResident(ctx, linearTerms, e0, &windowGraph(ctx, linearTerms, 0.0), 0.0));
        if (d_forces)
            IX_CUDA(ctx, cudaMemcpyAsync(dLin0, ctx->dOutForces, n3 * sizeof(double), cudaMemcpyDeviceToDevice,
                                         ctx->stream));
        ctx->parameters[name] = 1.0;
        IX_TRY(evaluateResident(ctx, linearTerms, e1, &windowGraph(ctx, linearTerms, 1.0), 1.0));
        if (d_forces && pairNonlinear)
            IX_CUDA(ctx, cudaMemcpyAsync(dLin1, ctx->dOutForces, n3 * sizeof(double), cudaMemcpyDeviceToDevice,
                                         ctx->stream));
        else dLin1 = ctx->dOutForces;
        pairs = ctx->lastPairs;
        triples = ctx->lastTriples;
    }
    // pair terms with a soft core: every window evaluated, back to back after the first
    std::vector<double> pairEnergy(4 * (size_t)num_windows, 0.0);
    if (pairNonlinear) {
        IX_TRY(prepare(ctx, pairTerms));
        for (int w = 0; w < num_windows; w++) {
            ctx->parameters[name] = values[w];
            if (w == 0) {
                double e[4];
                IX_TRY(evaluateResident(ctx, pairTerms, e, &windowGraph(ctx, pairTerms, values[w]), values[w]));
            }
            else IX_TRY(enqueueResident(ctx, pairTerms, windowGraph(ctx, pairTerms, values[w]), values[w]));
            IX_CUDA(ctx, cudaMemcpyAsync(dWinEnergy + 4 * (size_t)w, ctx->dOutEnergy, 4 * sizeof(double),
                                         cudaMemcpyDeviceToDevice, ctx->stream));
            if (d_forces)
                IX_CUDA(ctx, cudaMemcpyAsync(d_forces + w * n3, ctx->dOutForces, n3 * sizeof(double),
                                             cudaMemcpyDeviceToDevice, ctx->stream));
        }
        IX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        IX_TRY(checkOverflow(ctx, pairTerms, redo));
        if (redo) return IX_OK;
        IX_CUDA(ctx, cudaMemcpy(pairEnergy.data(), dWinEnergy, pairEnergy.size() * sizeof(double),
                                cudaMemcpyDeviceToHost));
        IX_TRY(readCounts(ctx, pairTerms));
        pairs = ctx->lastPairs;
    }
    ctx->lastPairs = pairs;
    ctx->lastTriples = triples;
    for (int w = 0; w < num_windows; w++)
        for (int k = 0; k < 4; k++)
            energies[4 * w + k] = pairEnergy[4 * (size_t)w + k] + e0[k] + values[w] * (e1[k] - e0[k]);
    if (d_forces) {
        if (linearTerms) {
            IX_TRY(stageCopy(ctx, dLambda, values, num_windows * sizeof(double)));
            const unsigned bx = (unsigned)std::max<size_t>(std::min<size_t>((n3 + 255) / 256, 1184), 1);
            const dim3 grid(bx, (unsigned)std::min(num_windows, 65535));
            kWindowForces<<<grid, 256, 0, ctx->stream>>>(n3, num_windows, dLambda, dLin0, dLin1, d_forces,
                                                         pairNonlinear ? 1 : 0);
            ctx->launches += 1;
            IX_CUDA(ctx, cudaGetLastError());
        }
        else if (!pairNonlinear)
            IX_CUDA(ctx, cudaMemsetAsync(d_forces, 0, num_windows * n3 * sizeof(double), ctx->stream));
        IX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return IX_OK;
}

// The context evaluated at several values of one alchemical parameter, forces left on the device (d_forces, n x 3
// per window, or null).  Terms whose alchemical scaling is linear in the parameter (pairs with exactly one
// alchemical particle and no soft core, triples with an alchemical site, the long-range correction coef + lambda
// alchCoef) are evaluated at 0 and 1 and interpolated for every window by kWindowForces; pair terms with a soft core
// (the alchemical pairs' distances depend on the parameter) are evaluated at every window, back to back.  Each value
// has its own cached graph, so repeated window sets replay without capturing.  The parameter keeps its value.
static int computeWindows(ix_ctx* ctx, const char* parameter, int num_windows, const double* values, double* energies,
                          double* d_forces) {
    NvtxRange nvtxRange("ix_compute_windows");
    if (!parameter || num_windows < 0 || (num_windows > 0 && (!values || !energies)))
        return fail(ctx, IX_ERR_INVALID, "ix_compute_windows: null argument");
    for (int w = 0; w < num_windows; w++)
        if (!std::isfinite(values[w])) return fail(ctx, IX_ERR_INVALID, "ix_compute_windows: window %d is not finite", w);
    if (num_windows == 0) return IX_OK;
    ctx->mdForcesValid = false;
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    const std::string name = parameter;
    const auto saved = ctx->parameters.find(name);
    const bool hadValue = saved != ctx->parameters.end();
    const double oldValue = hadValue ? saved->second : 0.0;
    int rc = IX_OK;
    for (int attempt = 0; attempt < 3; attempt++) {
        bool redo = false;
        rc = windowsPass(ctx, name, num_windows, values, energies, d_forces, redo);
        if (rc != IX_OK || !redo) break;
    }
    // the graphs of plain evaluations were captured with the old value: restoring it keeps them valid
    if (hadValue) ctx->parameters[name] = oldValue;
    else ctx->parameters.erase(name);
    return rc;
}

int ix_compute_windows_device(ix_ctx* ctx, const char* parameter, int num_windows, const double* values,
                              double* energies, double* d_forces) {
    if (!ctx) return IX_ERR_INVALID;
    return computeWindows(ctx, parameter, num_windows, values, energies, d_forces);
}

int ix_compute_windows(ix_ctx* ctx, const char* parameter, int num_windows, const double* values, double* energies,
                       double* forces) {
    if (!ctx) return IX_ERR_INVALID;
    double* dForces = nullptr;
    const size_t n3 = 3 * (size_t)ctx->n;
    if (forces && num_windows > 0) IX_TRY(deviceAlloc(ctx, "windowForces", (size_t)num_windows * n3, &dForces));
    IX_TRY(computeWindows(ctx, parameter, num_windows, values, energies, dForces));
    if (dForces)
        IX_CUDA(ctx, cudaMemcpy(forces, dForces, (size_t)num_windows * n3 * sizeof(double), cudaMemcpyDeviceToHost));
    return IX_OK;
}

int ix_get_launch_count(ix_ctx* ctx, long long* launches) {
    if (!ctx || !launches) return IX_ERR_INVALID;
    *launches = ctx->launches;
    return IX_OK;
}

// Finish enqueued MD steps: synchronize, check the neighbor lists, record the counts of the last evaluation, copy the
// state out.  When the pair list overflowed during the steps (their forces missed pairs), the list is grown, the
// state saved before the steps is restored and the steps are run again, as OpenMM recomputes a step whose neighbor
// list overflowed; a three-body list overflow needs no rerun (those sites scan every later site).
int ix_md_finish(ix_ctx* ctx, double* positions, double* velocities, double* energy) {
    NvtxRange nvtxRange("ix_md_finish");
    if (!ctx) return IX_ERR_INVALID;
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned terms = selectedTerms(ctx, -1);
    for (int attempt = 0;; attempt++) {
        IX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        bool redo = false;
        if (terms) IX_TRY(checkOverflow(ctx, terms, redo));
        if (!redo) break;
        if (ctx->mdPending.empty() || attempt == 4) {
            ctx->mdPending.clear();
            ctx->mdForcesValid = false;
            return fail(ctx, IX_ERR_STATE, "neighbor list overflow during MD; the lists were grown, rerun the steps");
        }
        IX_TRY(mdStateCopy(ctx, false));
        ctx->mdForcesValid = ctx->mdSavedForcesValid;
        // both lists are rebuilt from the restored positions (the pair list's flag is set by its growth), so that
        // the rerun is the run a large enough list gives, list for list
        if (ctx->atmAllocated) {
            const int one = 1;
            IX_CUDA(ctx, cudaMemcpy(ctx->dFlags + 4, &one, sizeof(int), cudaMemcpyHostToDevice));
        }
        for (const auto& seg : ctx->mdPending) IX_TRY(enqueueSteps(ctx, seg.first, seg.second));
        ctx->mdReruns++;
    }
    ctx->mdPending.clear();
    if (ctx->numConstraints) {
        int failed = 0;
        IX_CUDA(ctx, cudaMemcpy(&failed, ctx->K.fail, sizeof(int), cudaMemcpyDeviceToHost));
        if (failed) {
            const int zero = 0;
            IX_CUDA(ctx, cudaMemcpy(ctx->K.fail, &zero, sizeof(int), cudaMemcpyHostToDevice));
            return fail(ctx, IX_ERR_STATE, "the constraints did not converge during the MD steps");
        }
    }
    unsigned long long c[2] = {0, 0};
    IX_CUDA(ctx, cudaMemcpy(c, ctx->dCounts + 2, sizeof(c), cudaMemcpyDeviceToHost));
    ctx->lastPairs = (terms & 7u) ? (long long)c[0] : 0;
    ctx->lastTriples = (terms & 8u) ? (long long)c[1] : 0;
    const int n = ctx->n;
    if (positions)
        IX_CUDA(ctx, cudaMemcpy(positions, ctx->dPos, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    if (velocities)
        IX_CUDA(ctx, cudaMemcpy(velocities, ctx->dVel, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    if (energy) {
        double e[4] = {0, 0, 0, 0};
        if (terms) IX_CUDA(ctx, cudaMemcpy(e, ctx->dOutEnergy, sizeof(e), cudaMemcpyDeviceToHost));
        *energy = e[0] + e[1] + e[2] + e[3];
    }
    return IX_OK;
}

int ix_md_set_constraints(ix_ctx* ctx, int num_constraints, const int32_t* pairs, const double* distances,
                          double tolerance) {
    if (!ctx) return IX_ERR_INVALID;
    if (num_constraints < 0 || (num_constraints > 0 && (!pairs || !distances)))
        return fail(ctx, IX_ERR_INVALID, "ix_md_set_constraints: invalid arguments");
    if (!(tolerance > 0.0)) return fail(ctx, IX_ERR_INVALID, "ix_md_set_constraints: the tolerance must be positive");
    const int n = ctx->n;
    // clusters: the connected components of the constraint graph (union-find), single particles as their own
    std::vector<int> parent(n);
    for (int i = 0; i < n; i++) parent[i] = i;
    auto root = [&](int i) {
        while (parent[i] != i) i = parent[i] = parent[parent[i]];
        return i;
    };
    for (int k = 0; k < num_constraints; k++) {
        const int a = pairs[2 * k], b = pairs[2 * k + 1];
        if (a < 0 || b < 0 || a >= n || b >= n || a == b)
            return fail(ctx, IX_ERR_INVALID, "Illegal particle index for a constraint: %d, %d", a, b);
        if (!(distances[k] > 0.0)) return fail(ctx, IX_ERR_INVALID, "Illegal constraint distance: %g", distances[k]);
        const int ra = root(a), rb = root(b);
        if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
    }
    std::vector<int> clusterOf(n, -1), particleStart{0}, particles, members;
    std::vector<std::vector<int>> byRoot(n);
    for (int i = 0; i < n; i++) byRoot[root(i)].push_back(i);
    std::vector<int> local(n, 0);
    for (int r = 0; r < n; r++) {
        if (byRoot[r].empty()) continue;
        if ((int)byRoot[r].size() > kMaxClusterParticles)
            return fail(ctx, IX_ERR_INVALID, "a cluster of %zu constrained particles (the limit is %d)",
                        byRoot[r].size(), kMaxClusterParticles);
        const int c = (int)particleStart.size() - 1;
        for (size_t k = 0; k < byRoot[r].size(); k++) {
            clusterOf[byRoot[r][k]] = c;
            local[byRoot[r][k]] = (int)k;
            particles.push_back(byRoot[r][k]);
        }
        particleStart.push_back((int)particles.size());
    }
    const int numClusters = (int)particleStart.size() - 1;
    std::vector<std::vector<int>> consOf(numClusters);
    for (int k = 0; k < num_constraints; k++) consOf[clusterOf[pairs[2 * k]]].push_back(k);
    std::vector<int> consStart{0};
    std::vector<int2> pair;
    std::vector<double> dist2;
    for (int c = 0; c < numClusters; c++) {
        if ((int)consOf[c].size() > kMaxClusterConstraints)
            return fail(ctx, IX_ERR_INVALID, "a cluster of %zu constraints (the limit is %d)", consOf[c].size(),
                        kMaxClusterConstraints);
        const size_t first = pair.size();
        for (int k : consOf[c]) {
            pair.push_back(make_int2(local[pairs[2 * k]], local[pairs[2 * k + 1]]));
            dist2.push_back(distances[k] * distances[k]);
        }
        if (consOf[c].size() == 3 && particleStart[c + 1] - particleStart[c] == 3) {
            // a rigid triangle: its constraints as (0,1), (0,2), (1,2) (a constraint's orientation does not change
            // its solution), which the device solves with every index known at compile time
            std::vector<std::pair<int2, double>> tri;
            for (size_t q = first; q < pair.size(); q++) {
                const int2 e = pair[q];
                tri.push_back({make_int2(std::min(e.x, e.y), std::max(e.x, e.y)), dist2[q]});
            }
            std::sort(tri.begin(), tri.end(), [](const std::pair<int2, double>& a, const std::pair<int2, double>& b) {
                return a.first.x != b.first.x ? a.first.x < b.first.x : a.first.y < b.first.y;
            });
            if (tri[0].first.x == 0 && tri[0].first.y == 1 && tri[1].first.x == 0 && tri[1].first.y == 2 &&
                tri[2].first.x == 1 && tri[2].first.y == 2)
                for (int q = 0; q < 3; q++) {
                    pair[first + q] = tri[q].first;
                    dist2[first + q] = tri[q].second;
                }
        }
        consStart.push_back((int)pair.size());
    }
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    int *dPS, *dP, *dCS, *dFail;
    int2* dPair;
    double* dD2;
    IX_TRY(deviceAlloc(ctx, "clusterParticleStart", particleStart.size(), &dPS));
    IX_TRY(deviceAlloc(ctx, "clusterParticles", particles.size(), &dP));
    IX_TRY(deviceAlloc(ctx, "clusterConstraintStart", consStart.size(), &dCS));
    IX_TRY(deviceAlloc(ctx, "constraintPairs", std::max<size_t>(pair.size(), 1), &dPair));
    IX_TRY(deviceAlloc(ctx, "constraintDist2", std::max<size_t>(dist2.size(), 1), &dD2));
    IX_TRY(deviceAlloc(ctx, "constraintFail", 1, &dFail));
    IX_TRY(stageCopy(ctx, dPS, particleStart.data(), particleStart.size() * sizeof(int)));
    IX_TRY(stageCopy(ctx, dP, particles.data(), particles.size() * sizeof(int)));
    IX_TRY(stageCopy(ctx, dCS, consStart.data(), consStart.size() * sizeof(int)));
    if (!pair.empty()) {
        IX_TRY(stageCopy(ctx, dPair, pair.data(), pair.size() * sizeof(int2)));
        IX_TRY(stageCopy(ctx, dD2, dist2.data(), dist2.size() * sizeof(double)));
    }
    IX_CUDA(ctx, cudaMemsetAsync(dFail, 0, sizeof(int), ctx->stream));
    IX_TRY(uploadsDone(ctx));
    ctx->K = ConstraintClusters{numClusters, dPS, dP, dCS, dPair, dD2, tolerance, dFail};
    ctx->numConstraints = num_constraints;
    ctx->mdPending.clear();
    bumpVersion(ctx);
    return IX_OK;
}

int ix_md_run(ix_ctx* ctx, int num_steps, double dt, double* positions, double* velocities, double* energy) {
    if (!ctx) return IX_ERR_INVALID;
    if (!ctx->haveMasses) return fail(ctx, IX_ERR_STATE, "ix_md_run: masses have not been set");
    IX_CUDA(ctx, cudaSetDevice(ctx->device));
    if (velocities)
        IX_TRY(stageCopy(ctx, ctx->dVel, velocities, 3 * (size_t)ctx->n * sizeof(double)));
    IX_TRY(ix_md_steps_async(ctx, num_steps, dt));
    return ix_md_finish(ctx, positions, velocities, energy);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------------
// Three-body evaluation without any allocation.
//
// Some callers cannot call cudaMalloc at the point where they need the forces: a CUDA graph being captured (an
// allocation inside stream capture is not allowed), an engine whose device memory is owned by its own pool, or a
// real-time loop that must not allocate.  For them ix_three_body_noalloc evaluates the three-body force with all its
// working memory in one file-scope __device__ array of fixed size; the caller passes only its inputs and outputs.
// Limits: kNoAllocMaxParticles particles, kNoAllocMaxSites sites; a site with more than kNoAllocMaxNeighbors sites
// above it within the cutoff is evaluated by a scan of every later site (reported by the overflow query).  The array is allocated by the CUDA runtime when the library is loaded, on every GPU that loads it
// (about 2.7 MB), and stays until the process exits.  Every call shares it: two calls that overlap on the GPU (on
// different streams, or from different host threads on one device) race on it and must be serialized by the caller.
// ---------------------------------------------------------------------------------------------------------------------

namespace {

constexpr int kNoAllocMaxParticles = 16384;
constexpr int kNoAllocMaxSites = 4096;
constexpr int kNoAllocMaxNeighbors = 128;
constexpr int kNoAllocFastBlocks = kNoAllocMaxSites / kAtmFastWarps;   // one warp per site
constexpr int kNoAllocBlocks = 148 * 2;                                 // grid of the wide triple kernel

struct NoAllocScratch {
    double sitePos[3 * kNoAllocMaxSites];
    double siteRef[3 * kNoAllocMaxSites];
    float4 siteParams[kNoAllocMaxSites];
    int molecule[kNoAllocMaxSites];
    int nbrCount[kNoAllocMaxSites];
    int nbr[kNoAllocMaxSites * kNoAllocMaxNeighbors];
    long long siteForce[3 * kNoAllocMaxSites];
    long long particleForce[3 * kNoAllocMaxParticles];
    double energyPartials[kNoAllocFastBlocks * kAtmFastWarps + kNoAllocBlocks * kAtmWarps];
    double energy[4];
    double energyBlocks[4];      // the energy reduction's block sum (one block)
    unsigned reduceTicket;
    int flag[3];
    unsigned long long tripleCount;
};

// The scratch itself.  Host code must not use this name as a pointer: on the host it is only a stand-in for the
// symbol, and its device address comes from cudaGetSymbolAddress (noAllocScratch() below).
__device__ __align__(256) unsigned char g_noAllocScratch[sizeof(NoAllocScratch)];

constexpr int kMaxDevices = 64;
void* g_noAllocAddress[kMaxDevices] = {};
std::mutex g_noAllocMutex;

// Device address of the scratch on the current device, looked up once per device.
int noAllocScratch(int device, NoAllocScratch** out) {
    if (device < 0 || device >= kMaxDevices) return fail(nullptr, IX_ERR_NO_DEVICE, "device index %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noAllocMutex);
    if (!g_noAllocAddress[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noAllocScratch);
        if (e != cudaSuccess)
            return fail(nullptr, IX_ERR_CUDA, "cudaGetSymbolAddress of the three-body scratch failed: %s",
                        cudaGetErrorString(e));
        g_noAllocAddress[device] = p;
    }
    *out = reinterpret_cast<NoAllocScratch*>(g_noAllocAddress[device]);
    return IX_OK;
}

// Per call: site parameters in the kernels' layout, the effective molecules, and the accumulators cleared.
__global__ void kNoAllocPrepare(NoAllocScratch* S, int numParticles, int numSites, const double* siteParams,
                                const int* molecule, const uint8_t* alch) {
    const int stride = gridDim.x * blockDim.x;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    for (int s = t; s < numSites; s += stride) {
        S->siteParams[s] = make_float4((float)siteParams[3 * s], (float)siteParams[3 * s + 1],
                                       (float)siteParams[3 * s + 2], alch[s] ? 1.0f : 0.0f);
        S->molecule[s] = molecule[s] < 0 ? -1 - s : molecule[s];
        for (int d = 0; d < 3; d++) {
            S->siteForce[d * numSites + s] = 0;
            S->siteRef[3 * s + d] = 0.0;
        }
    }
    for (int i = t; i < 3 * numParticles; i += stride) S->particleForce[i] = 0;
    if (t == 0) {
        S->flag[0] = 1;      // always build the neighbor list
        S->flag[1] = 0;
        S->flag[2] = 0;
        S->tripleCount = 0;
    }
}

// Site positions with the particle indices checked (an index outside [0, numParticles) is skipped).
__global__ void kNoAllocCentroids(NoAllocScratch* S, int numParticles, int numSites, const int* offsets,
                                  const int* particles, const double* pos) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= numSites) return;
    double c[3] = {0.0, 0.0, 0.0};
    int count = 0;
    for (int k = offsets[s]; k < offsets[s + 1]; k++) {
        const int p = particles[k];
        if (p < 0 || p >= numParticles) continue;
        for (int d = 0; d < 3; d++) c[d] += pos[3 * p + d];
        count++;
    }
    for (int d = 0; d < 3; d++) S->sitePos[3 * s + d] = count ? c[d] / (double)count : 0.0;
}

__global__ void kNoAllocSpread(NoAllocScratch* S, int numParticles, int numSites, const int* offsets,
                               const int* particles) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= numSites) return;
    const int b = offsets[s], e = offsets[s + 1];
    int count = 0;
    for (int k = b; k < e; k++) count += (particles[k] >= 0 && particles[k] < numParticles);
    if (!count) return;
    const double inv = 1.0 / (double)count;
    for (int d = 0; d < 3; d++) {
        const long long v = S->siteForce[d * numSites + s];
        if (v == 0) continue;
        const long long share = __double2ll_rn((double)v * inv);
        for (int k = b; k < e; k++) {
            const int p = particles[k];
            if (p >= 0 && p < numParticles) atomicAddFixed(S->particleForce + (size_t)d * numParticles + p, share);
        }
    }
}

__global__ void kNoAllocFinish(const NoAllocScratch* S, int numParticles, double* forces) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numParticles) return;
    for (int d = 0; d < 3; d++)
        forces[3 * i + d] = (double)S->particleForce[(size_t)d * numParticles + i] / kFixedScale;
}

}  // namespace

extern "C" {

int ix_three_body_noalloc(int num_particles, const double* d_positions, const double* box, int num_sites,
                          const int32_t* d_site_offsets, const int32_t* d_site_particles,
                          const double* d_site_params, const int32_t* d_molecule, const uint8_t* d_is_alchemical,
                          double cutoff, double scale_factor, int damping_method, double damping_scale,
                          double centroid_damping_radius, int periodic, double lambda, double* d_forces,
                          double* d_energy, void* stream) {
    NvtxRange nvtxRange("ix_three_body_noalloc");
    if (num_particles <= 0 || num_particles > kNoAllocMaxParticles)
        return fail(nullptr, IX_ERR_INVALID, "ix_three_body_noalloc: %d particles (the limit is %d)", num_particles,
                    kNoAllocMaxParticles);
    if (num_sites < 0 || num_sites > kNoAllocMaxSites)
        return fail(nullptr, IX_ERR_INVALID, "ix_three_body_noalloc: %d sites (the limit is %d)", num_sites,
                    kNoAllocMaxSites);
    if (!d_positions || !d_forces || !d_energy || (num_sites > 0 && (!d_site_offsets || !d_site_particles ||
                                                                     !d_site_params || !d_molecule ||
                                                                     !d_is_alchemical)))
        return fail(nullptr, IX_ERR_INVALID, "ix_three_body_noalloc: null argument");
    if (periodic && !box) return fail(nullptr, IX_ERR_INVALID, "ix_three_body_noalloc: periodic without a box");
    if (damping_method != IX_NO_DAMPING && damping_method != IX_TANG_TOENNIES)
        return fail(nullptr, IX_ERR_INVALID, "InteraxThreeBodyForce: Illegal value for damping method");
    if (cutoff <= 0) return fail(nullptr, IX_ERR_INVALID, "InteraxThreeBodyForce: The cutoff distance must be positive");
    if (centroid_damping_radius < 0)
        return fail(nullptr, IX_ERR_INVALID, "InteraxThreeBodyForce: The centroid damping radius cannot be negative");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_NO_DEVICE, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    NoAllocScratch* S = nullptr;
    IX_TRY(noAllocScratch(device, &S));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int tpb = 256;
    kNoAllocPrepare<<<64, tpb, 0, st>>>(S, num_particles, num_sites, d_site_params, d_molecule, d_is_alchemical);
    kNoAllocCentroids<<<(num_sites + tpb - 1) / tpb + 1, tpb, 0, st>>>(S, num_particles, num_sites, d_site_offsets,
                                                                      d_site_particles, d_positions);
    AtmConfig C{};
    C.numSites = num_sites;
    C.periodic = periodic != 0;
    double unit[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    C.box = makeBox(box ? box : unit);
    C.boxf = makeBoxF(C.box);
    C.cutoff2 = (float)(cutoff * cutoff);
    C.listCutoff2 = C.cutoff2;
    C.scale = (float)scale_factor;
    C.lambda = (float)lambda;
    C.useTangToennies = damping_method == IX_TANG_TOENNIES;
    C.twoBeta = (float)(2.0 * damping_scale);
    C.invCentroidRadius = centroid_damping_radius > 0 ? (float)(1.0 / centroid_damping_radius) : 0.0f;
    C.maxMove2 = 0.0f;
    AtmBuffers A{};
    A.siteParams = S->siteParams;
    A.molecule = S->molecule;
    A.sitePos = S->sitePos;
    A.siteRef = S->siteRef;
    A.flag = S->flag;
    A.nbrCount = S->nbrCount;
    A.nbr = S->nbr;
    A.cap = kNoAllocMaxNeighbors;
    A.siteForce = S->siteForce;
    A.particleForce = S->particleForce;
    A.numParticles = num_particles;
    A.energyPartials = S->energyPartials;
    A.tripleCount = &S->tripleCount;
    if (num_sites > 0) {
        kSiteNeighbors<<<(num_sites * 32 + tpb - 1) / tpb, tpb, 0, st>>>(A, C);
        const int fastBlocks = (num_sites + kAtmFastWarps - 1) / kAtmFastWarps;
        const int blocks = std::max(1, std::min((num_sites + kAtmWarps - 1) / kAtmWarps, kNoAllocBlocks));
        kTriplesFast<<<fastBlocks, 32 * kAtmFastWarps, 0, st>>>(A, C);
        kTriplesWide<<<blocks, 32 * kAtmWarps, sizeof(AtmWarpStorage) * kAtmWarps, st>>>(A, C,
                                                                                        fastBlocks * kAtmFastWarps,
                                                                                        nullptr);
        kNoAllocSpread<<<(num_sites + tpb - 1) / tpb, tpb, 0, st>>>(S, num_particles, num_sites, d_site_offsets,
                                                                   d_site_particles);
        kReduceEnergies<<<1, 256, 0, st>>>(nullptr, nullptr, 0, S->energyPartials,
                                           fastBlocks * kAtmFastWarps + blocks * kAtmWarps, 0.0, S->energy,
                                           S->energyBlocks, &S->reduceTicket, nullptr, nullptr);
    }
    else {
        kReduceEnergies<<<1, 256, 0, st>>>(nullptr, nullptr, 0, nullptr, 0, 0.0, S->energy, S->energyBlocks,
                                           &S->reduceTicket, nullptr, nullptr);
    }
    kNoAllocFinish<<<(num_particles + tpb - 1) / tpb, tpb, 0, st>>>(S, num_particles, d_forces);
    e = cudaMemcpyAsync(d_energy, &S->energy[3], sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_CUDA, "ix_three_body_noalloc: %s", cudaGetErrorString(e));
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_CUDA, "ix_three_body_noalloc: %s", cudaGetErrorString(e));
    return IX_OK;
}

int ix_three_body_noalloc_overflow(int* overflow) {
    if (!overflow) return fail(nullptr, IX_ERR_INVALID, "ix_three_body_noalloc_overflow: null argument");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_NO_DEVICE, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    NoAllocScratch* S = nullptr;
    IX_TRY(noAllocScratch(device, &S));
    // the flag is written by the last call's kernels on the caller's stream, which may be a non-blocking stream that a
    // plain copy does not wait for: wait for the whole device first
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_CUDA, "ix_three_body_noalloc_overflow: %s", cudaGetErrorString(e));
    int flags[2] = {0, 0};
    e = cudaMemcpy(flags, S->flag, sizeof(flags), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(nullptr, IX_ERR_CUDA, "ix_three_body_noalloc_overflow: %s", cudaGetErrorString(e));
    *overflow = flags[1] != 0;
    return IX_OK;
}

}  // extern "C"

// batched evaluation of many small systems (its own translation-unit part; reuses the helpers above)
#include "ix_batch.cuh"
#include "ix_server.cuh"
