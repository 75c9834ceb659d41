// A request server: continuous batching of independent energy+force / MD requests of mixed sizes on one GPU.
// Included at the end of ix_context.cu (after ix_batch.cuh), whose contexts and batches it runs.
//
// Native worker threads (shards) own the device side; each runs its own requests (small requests all go to shard 0,
// so that they gather into large cohorts; periodic requests are spread over all shards, whose host work of launching
// them then proceeds in parallel).  Each pass of a shard's loop
//   1. moves newly submitted requests into the shard's pending queue (FIFO),
//   2. admits pending requests while the running count and the device memory budget allow (a request whose estimate
//      does not fit waits; later, smaller requests may pass it), launching each admitted periodic request as a
//      context on its own streams and gathering admitted small non-periodic requests into a cohort (an ix_batch run
//      with per-system step counts, one CUDA graph per MD step of the whole cohort),
//   3. checks the events that mark finished requests: their results were copied by their own stream into pinned
//      staging, so the worker only unpacks them, and frees the unit's memory when its last request is done.
// All launches are asynchronous, so every admitted request's work overlaps on the device.  Device memory comes from one
// arena bounded by the budget; the estimate of each request is reserved atomically at admission, so shards never
// over-commit it.  A context's streams and events go back to its shard's pool and its CUDA graphs to a reaper thread
// when it finishes, so that no teardown call of the worker waits for the device.  A request's state
// (positions, velocities, parameters, neighbor lists) stays resident on the device from admission to its last step.
// Its results are those of the same request run alone: a context runs the same kernels either way, and a batched
// system's evaluation is independent of the other systems of its batch.
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

namespace {

double serverNow() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Adds the seconds of its scope to one of the worker's time counters.
struct PhaseTimer {
    double& total;
    double t0;
    explicit PhaseTimer(double& t) : total(t), t0(serverNow()) {}
    ~PhaseTimer() { total += serverNow() - t0; }
};

// Host memory that the device can copy into asynchronously: chunks from cudaHostAlloc, sub-allocated best fit.
struct PinnedPool {
    std::mutex m;
    std::vector<char*> chunks;
    RangeHeap heap;
    size_t chunkBytes = size_t(256) << 20;

    char* alloc(size_t bytes) {
        bytes = (std::max<size_t>(bytes, 1) + 255) / 256 * 256;
        std::lock_guard<std::mutex> lock(m);
        char* p = heap.take(bytes);
        if (p) return p;
        char* base = nullptr;
        const size_t want = std::max(chunkBytes, bytes);
        if (cudaHostAlloc(reinterpret_cast<void**>(&base), want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        chunks.push_back(base);
        heap.addFree(base, want, (int)chunks.size() - 1);
        return heap.take(bytes);
    }

    void release(char* p) {
        std::lock_guard<std::mutex> lock(m);
        heap.give(p);
    }

    ~PinnedPool() {
        for (char* c : chunks) cudaFreeHost(c);
    }
};

struct ServerRequest {
    long long id = 0;
    ix_ctx* sys = nullptr;               // the description; becomes the device context of a periodic request
    std::vector<double> pos, vel, mass;  // starting state, replaced by the final state
    std::vector<double> forces;
    double energies[4] = {0, 0, 0, 0};
    int steps = 0;
    double dt = 0.0;
    double tSubmit = 0.0, tDone = 0.0;
    size_t estimate = 0;
    bool small = false;
    std::string desc;                    // a periodic request's System, serialized: the key of the context pool
    unsigned long long key = 0;          // its hash
    int status = IX_OK;
    std::string error;
};

// An admitted unit of work: one request's context, or a cohort of small requests in one batch.
struct ServerUnit {
    ix_ctx* ctx = nullptr;
    ix_batch* batch = nullptr;
    std::vector<ServerRequest*> members;  // a cohort's members in batch order (ascending steps)
    struct Mark {
        cudaEvent_t event = nullptr;
        int first = 0, last = 0;          // members [first, last) are complete when the event is
    };
    std::vector<Mark> marks;
    size_t next = 0;
    char* staging = nullptr;             // pinned copies of the results, written by the unit's stream
    size_t reserved = 0;                 // device bytes reserved for the unit (its actual bytes once launched)
    int restarts = 0;
};

// A context's streams and events, kept for the next context of the shard.
struct StreamSet {
    cudaStream_t stream = nullptr, stream2 = nullptr, body = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

// A context whose request finished, kept with its device arrays, streams and CUDA graphs for the next request of the
// same System (the same particles, forces, parameters and masses; only the state differs).
struct PooledContext {
    ix_ctx* ctx = nullptr;
    std::string desc;
    size_t reserved = 0;                 // device bytes it holds, still reserved against the budget
    double lastUse = 0.0;
};

struct ServerShard {
    int index = 0;
    std::unordered_multimap<unsigned long long, PooledContext> pool;
    size_t poolBytes = 0;
    std::thread worker;
    std::deque<ServerRequest*> incoming;     // guarded by the server's mutex
    std::deque<ServerRequest*> pending;
    std::vector<ServerUnit*> units;
    std::vector<cudaEvent_t> freeEvents;
    std::vector<StreamSet> streams;
    std::vector<cudaStream_t> cohortStreams;
    long long running = 0;
    double workerSec[12] = {};           // see ix_server_stats::worker_seconds
};

}  // namespace

struct ix_server {
    int device = 0;
    int numSMs = 148;
    DeviceArena arena;
    PinnedPool pinned;
    double budget = 0.0;
    std::atomic<long long> reserved{0};      // device bytes reserved by admitted units, all shards
    std::atomic<long long> peakReserved{0};
    int maxRunning = 256;                    // per shard
    int smallAtoms = 1024;
    int maxCohort = 512;
    double window = 200e-6;
    std::vector<std::unique_ptr<ServerShard>> shards;
    size_t maxPooled = 64;                   // idle contexts kept per shard for reuse
    std::mutex m;                        // guards the shards' incoming queues, done, doneIds, error, stats, stop
    std::condition_variable cvSubmit, cvDone;
    bool stop = false;
    std::map<long long, ServerRequest*> done;
    std::deque<long long> doneIds;
    long long nextId = 1;
    size_t nextShard = 0;
    std::string error;
    ix_server_stats stats{};
    // CUDA graphs of finished contexts, destroyed by the reaper thread
    std::thread reaper;
    std::mutex graveM;
    std::condition_variable graveCv;
    std::deque<cudaGraphExec_t> grave;
    bool graveStop = false;
};

namespace {

// A periodic request's System serialized for the context pool: everything a context's device arrays and graphs
// depend on (particle count, box, masses, parameter values, every force's settings and per-particle parameters,
// exclusions, sites), so that equal strings mean a context can be reused as it is.
template <class T>
void putBytes(std::string& out, const T* p, size_t count) {
    out.append(reinterpret_cast<const char*>(p), count * sizeof(T));
}
template <class T>
void putValue(std::string& out, const T& v) {
    putBytes(out, &v, 1);
}
template <class T>
void putVector(std::string& out, const std::vector<T>& v) {
    putValue(out, v.size());
    putBytes(out, v.data(), v.size());
}

std::string poolDescription(const ix_ctx* c, const std::vector<double>& mass) {
    std::string d;
    putValue(d, c->n);
    putBytes(d, c->box, 9);
    putVector(d, mass);
    for (const auto& kv : c->parameters) {
        d += kv.first;
        putValue(d, kv.second);
    }
    putValue(d, c->method);
    putValue(d, c->cutoff);
    putValue(d, c->exclusions.size());
    for (const auto& e : c->exclusions) {
        putValue(d, e.first);
        putValue(d, e.second);
    }
    for (const PairTerm& T : c->term) {
        putValue(d, T.present);
        if (!T.present) continue;
        putValue(d, T.group);
        d += T.alchName;
        putValue(d, T.useSwitch);
        putValue(d, T.switchDistance);
        putValue(d, T.softcoreRadius);
        putValue(d, T.overlapMethod);
        putValue(d, T.dampingScale);
        putValue(d, T.useLrc);
        putVector(d, T.params);
        putVector(d, T.alch);
    }
    putValue(d, c->atmPresent);
    if (c->atmPresent) {
        putValue(d, c->atmGroup);
        d += c->atmAlchName;
        putVector(d, c->siteOffsets);
        putVector(d, c->siteParticles);
        putVector(d, c->molecule);
        putVector(d, c->siteParams);
        putVector(d, c->siteAlch);
        putValue(d, c->atmCutoff);
        putValue(d, c->atmScale);
        putValue(d, c->atmDampingScale);
        putValue(d, c->atmCentroidRadius);
        putValue(d, c->atmDamping);
        putValue(d, c->atmPeriodic);
    }
    return d;
}

// FNV-1a, 64 bits.
unsigned long long hashBytes(const std::string& s) {
    unsigned long long h = 1469598103934665603ull;
    for (unsigned char ch : s) {
        h ^= ch;
        h *= 1099511628211ull;
    }
    return h;
}

// Device bytes a request will hold, an upper bound used for admission (the unit's actual bytes replace it once it
// is launched).  A periodic context holds per-particle arrays, the pair tiles (a few hundred bytes per tile, ~75 tiles
// per 32-particle block at water density and a 1 nm cutoff, with the list's growth margin) and the three-body site
// lists; a batched system holds its all-pairs block tiles and all-sites lists.
size_t estimateRequestBytes(const ix_ctx* c, bool small) {
    const size_t n = (size_t)c->n, sites = c->siteParams.size() / 3, nb = (n + 31) / 32;
    if (small) return (size_t(64) << 10) + 1024 * n + 640 * (nb * (nb + 1) / 2) + 16 * sites * sites + 512 * sites;
    return (size_t(8) << 20) + 6144 * n + 4096 * sites;
}

// Reserve device bytes against the budget; false if they do not fit.
bool reserveBytes(ix_server* S, size_t bytes) {
    const long long b = (long long)bytes;
    long long cur = S->reserved.load();
    while ((double)(cur + b) <= S->budget)
        if (S->reserved.compare_exchange_weak(cur, cur + b)) {
            long long peak = S->peakReserved.load();
            while (cur + b > peak && !S->peakReserved.compare_exchange_weak(peak, cur + b)) {
            }
            return true;
        }
    return false;
}

void unreserveBytes(ix_server* S, size_t bytes) { S->reserved -= (long long)bytes; }

void retireContext(ix_server* S, ServerShard* H, ix_ctx* c);

// An idle context of the shard's pool for request r (nullptr: none), taken out of the pool.
PooledContext takePooled(ServerShard* H, const ServerRequest* r) {
    auto range = H->pool.equal_range(r->key);
    for (auto it = range.first; it != range.second; ++it)
        if (it->second.desc == r->desc) {
            PooledContext p = std::move(it->second);
            H->pool.erase(it);
            H->poolBytes -= p.reserved;
            return p;
        }
    return PooledContext{};
}

bool hasPooled(const ServerShard* H, const ServerRequest* r) {
    auto range = H->pool.equal_range(r->key);
    for (auto it = range.first; it != range.second; ++it)
        if (it->second.desc == r->desc) return true;
    return false;
}

// Retire the shard's least recently used idle context; false when the pool is empty.
bool evictPooled(ix_server* S, ServerShard* H) {
    if (H->pool.empty()) return false;
    auto oldest = H->pool.begin();
    for (auto it = H->pool.begin(); it != H->pool.end(); ++it)
        if (it->second.lastUse < oldest->second.lastUse) oldest = it;
    PooledContext p = std::move(oldest->second);
    H->pool.erase(oldest);
    H->poolBytes -= p.reserved;
    retireContext(S, H, p.ctx);
    unreserveBytes(S, p.reserved);
    return true;
}

size_t bufferBytes(const std::map<std::string, DeviceBuffer>& buffers) {
    size_t total = 0;
    for (const auto& kv : buffers) total += kv.second.bytes;
    return total;
}

cudaEvent_t shardEvent(ServerShard* H) {
    if (!H->freeEvents.empty()) {
        cudaEvent_t e = H->freeEvents.back();
        H->freeEvents.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
}

void serverFinish(ix_server* S, ServerShard* H, ServerRequest* r, int status, const std::string& error) {
    r->tDone = serverNow();
    r->status = status;
    r->error = error;
    if (r->sys) {
        ix_ctx_destroy(r->sys);
        r->sys = nullptr;
    }
    {
        std::lock_guard<std::mutex> lock(S->m);
        S->done[r->id] = r;
        S->doneIds.push_back(r->id);
        if (status == IX_OK) S->stats.completed++;
        else S->stats.failed++;
    }
    if (H) H->running--;
    S->cvDone.notify_all();
}

// Destroy a finished context without waiting for the device: its streams and events go back to the shard's pool,
// its graphs to the reaper, its memory to the arena.
void retireContext(ix_server* S, ServerShard* H, ix_ctx* c) {
    if (c->stream) cudaStreamSynchronize(c->stream);   // idle already: its last event has completed
    StreamSet set;
    set.stream = c->stream;
    set.stream2 = c->stream2;
    set.body = c->streamBody;
    set.fork = c->evFork;
    set.join = c->evJoin;
    if (set.stream && set.stream2 && set.body && set.fork && set.join) {
        H->streams.push_back(set);
        c->stream = c->stream2 = c->streamBody = nullptr;
        c->evFork = c->evJoin = nullptr;
    }
    {
        std::lock_guard<std::mutex> lock(S->graveM);
        for (LaunchGraph* g : {&c->graphCompute, &c->graphDevice, &c->graphMd})
            if (g->exec) {
                S->grave.push_back(g->exec);
                g->exec = nullptr;
            }
        for (auto& g : c->graphWindows)
            if (g.exec) {
                S->grave.push_back(g.exec);
                g.exec = nullptr;
            }
    }
    S->graveCv.notify_one();
    ix_ctx_destroy(c);
}

void reaperLoop(ix_server* S) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lock(S->graveM);
    for (;;) {
        S->graveCv.wait(lock, [&] { return S->graveStop || !S->grave.empty(); });
        if (S->grave.empty() && S->graveStop) break;
        cudaGraphExec_t g = S->grave.front();
        S->grave.pop_front();
        lock.unlock();
        cudaGraphExecDestroy(g);
        lock.lock();
    }
}

// Requests with at least this many steps run each step as one CUDA graph (the capture costs about a millisecond);
// shorter ones launch their kernels directly.
#ifndef IX_SERVER_GRAPH_STEPS
#define IX_SERVER_GRAPH_STEPS 16
#endif
constexpr int kServerGraphSteps = IX_SERVER_GRAPH_STEPS;

// Enqueue a periodic request's whole run on its context's stream: positions, masses and velocities in, the first
// evaluation and every step, then the final state copied into the pinned staging, and the event that marks it done.
int enqueueContextRun(ServerShard* H, ServerUnit* u, bool reused = false) {
    ServerRequest* r = u->members[0];
    ix_ctx* c = u->ctx;
    const size_t n3 = 3 * (size_t)c->n;
    {
        PhaseTimer t(H->workerSec[10]);
        IX_TRY(ix_set_positions(c, r->pos.data(), nullptr));
        if (r->mass.empty()) r->mass.assign(c->n, 1.0);
        // a pooled context has these masses already (they are part of its description); setting them again would
        // invalidate its CUDA graphs
        if (!reused) IX_TRY(ix_md_set_masses(c, r->mass.data()));
        // both neighbor lists are rebuilt from the starting positions (a pooled context or a rerun after an overflow
        // holds lists of other positions), so that the request runs exactly as on a new context
        const int rebuild = 1;
        IX_TRY(stageCopy(c, c->dFlags, &rebuild, sizeof(int)));
        if (c->atmAllocated) IX_TRY(stageCopy(c, c->dFlags + 4, &rebuild, sizeof(int)));
        if (r->vel.empty()) IX_CUDA(c, cudaMemsetAsync(c->dVel, 0, n3 * sizeof(double), c->stream));
        else IX_TRY(stageCopy(c, c->dVel, r->vel.data(), n3 * sizeof(double)));
    }
    c->mdForcesValid = false;
    {
        PhaseTimer t(H->workerSec[11]);
        IX_TRY(ix_md_steps_async(c, r->steps, r->dt));
    }
    double* st = reinterpret_cast<double*>(u->staging);
    IX_CUDA(c, cudaMemcpyAsync(st, c->dPos, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    IX_CUDA(c, cudaMemcpyAsync(st + n3, c->dVel, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    IX_CUDA(c, cudaMemcpyAsync(st + 2 * n3, c->dOutForces, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    IX_CUDA(c, cudaMemcpyAsync(st + 3 * n3, c->dOutEnergy, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    IX_CUDA(c, cudaMemcpyAsync(st + 3 * n3 + 4, c->dFlags, 8 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ServerUnit::Mark mk;
    mk.event = shardEvent(H);
    mk.first = 0;
    mk.last = 1;
    IX_CUDA(c, cudaEventRecord(mk.event, c->stream));
    u->marks.assign(1, mk);
    u->next = 0;
    return IX_OK;
}

// Launch an admitted periodic request (its estimate already reserved): its description becomes a device context in
// the server's arena, with streams from the shard's pool.
void launchContext(ix_server* S, ServerShard* H, ServerRequest* r) {
    ServerUnit* u = new ServerUnit();
    u->members.push_back(r);
    u->reserved = r->estimate;
    {
        // an idle context of the same System: its arrays, lists and graphs are reused, only the state is uploaded
        PooledContext p = takePooled(H, r);
        if (p.ctx) {
            int rc = IX_OK;
            ix_ctx_destroy(r->sys);         // the description is no longer needed
            r->sys = p.ctx;
            u->ctx = p.ctx;
            unreserveBytes(S, u->reserved);   // the pooled context's bytes are reserved already
            u->reserved = p.reserved;
            p.ctx->useGraphs = r->steps >= kServerGraphSteps;
            {
                PhaseTimer t(H->workerSec[0]);
                const size_t results = (9 * (size_t)p.ctx->n + 8) * sizeof(double);
                u->staging = S->pinned.alloc(results + 320 * (size_t)p.ctx->n + (size_t(64) << 10));
                if (!u->staging) rc = fail(p.ctx, IX_ERR_MEMORY, "pinned host staging could not be allocated");
                else {
                    p.ctx->uploadBuf = u->staging + results;
                    p.ctx->uploadCap = 320 * (size_t)p.ctx->n + (size_t(64) << 10);
                    p.ctx->uploadUsed = 0;
                }
            }
            if (rc == IX_OK) {
                PhaseTimer t(H->workerSec[1]);
                rc = enqueueContextRun(H, u, true);
            }
            if (rc != IX_OK) {
                const std::string msg = p.ctx->error;
                for (auto& mk : u->marks) H->freeEvents.push_back(mk.event);
                if (u->staging) S->pinned.release(u->staging);
                r->sys = nullptr;
                retireContext(S, H, p.ctx);
                unreserveBytes(S, u->reserved);
                delete u;
                serverFinish(S, H, r, rc, msg);
                return;
            }
            H->units.push_back(u);
            std::lock_guard<std::mutex> lock(S->m);
            S->stats.contexts++;
            S->stats.contexts_reused++;
            S->stats.admitted++;
            return;
        }
    }
    ix_ctx* c = r->sys;
    c->arena = &S->arena;
    c->device = S->device;
    c->useGraphs = r->steps >= kServerGraphSteps;
    c->mdRollback = false;   // an overflow reruns the whole request from its description
    if (!H->streams.empty()) {
        const StreamSet set = H->streams.back();
        H->streams.pop_back();
        c->stream = set.stream;
        c->stream2 = set.stream2;
        c->streamBody = set.body;
        c->evFork = set.fork;
        c->evJoin = set.join;
    }
    u->ctx = c;
    int rc;
    {
        PhaseTimer t(H->workerSec[0]);
        // pinned staging: the results, then every upload of the request (parameters, lists, state)
        const size_t results = (9 * (size_t)c->n + 8) * sizeof(double);
        const size_t uploads = 320 * (size_t)c->n + 64 * (c->siteParams.size() / 3) + 8 * c->exclusions.size() +
                               (size_t(64) << 10);
        {
            PhaseTimer tp(H->workerSec[8]);
            u->staging = S->pinned.alloc(results + uploads);
        }
        rc = IX_OK;
        if (!u->staging) rc = fail(c, IX_ERR_MEMORY, "pinned host staging could not be allocated");
        else {
            c->uploadBuf = u->staging + results;
            c->uploadCap = uploads;
            c->uploadUsed = 0;
            PhaseTimer td(H->workerSec[9]);
            rc = ctxInitDevice(c);
        }
    }
    if (rc == IX_OK) {
        PhaseTimer t(H->workerSec[1]);
        rc = enqueueContextRun(H, u);
    }
    if (rc != IX_OK) {
        const std::string msg = c->error;
        for (auto& mk : u->marks) H->freeEvents.push_back(mk.event);
        if (u->staging) S->pinned.release(u->staging);
        r->sys = nullptr;
        retireContext(S, H, c);
        unreserveBytes(S, u->reserved);
        delete u;
        serverFinish(S, H, r, rc, msg);
        return;
    }
    // a context that holds more than its estimate reserves the difference too
    const size_t actual = bufferBytes(c->buffers);
    if (actual > u->reserved) {
        S->reserved += (long long)(actual - u->reserved);
        u->reserved = actual;
    }
    H->units.push_back(u);
    std::lock_guard<std::mutex> lock(S->m);
    S->stats.contexts++;
    S->stats.admitted++;
}

// Whether a small request can join a cohort started by r0: the same force settings, parameters and step size, and a
// size within a factor of kCohortSizeBand of r0's.  A cohort advances all its members step by step, so a small
// request beside a large one (whose all-pairs and all-triples cost grows as n^2 and n^3) would wait for the large
// one's steps.
constexpr int kCohortSizeBand = 2;
bool cohortCompatible(const ServerRequest* r, const ServerRequest* r0) {
    const int a = std::min(r->sys->n, r0->sys->n), b = std::max(r->sys->n, r0->sys->n);
    return b <= kCohortSizeBand * a && r->dt == r0->dt && r->sys->parameters == r0->sys->parameters &&
           sameBatchSettings(r->sys, r0->sys);
}

// Enqueue a cohort's whole run on its batch's stream: the first evaluation, then every step up to the longest
// request; after the last step of each group of requests (members are ordered by steps) their final state is copied
// into the pinned staging and an event marks them done.
// The members' starting state (positions, velocities, masses and step counts) for the cohort's batch, held with the
// build's uploads (the batch defers them).
int stageCohortState(ServerUnit* u) {
    ix_batch* b = u->batch;
    const int nm = (int)u->members.size(), np = b->numParticles;
    std::vector<double> pos(3 * (size_t)np), vel(3 * (size_t)np, 0.0), mass((size_t)np, 1.0);
    std::vector<int> steps(nm);
    for (int k = 0; k < nm; k++) {
        const ServerRequest* r = u->members[k];
        const size_t p0 = (size_t)b->particleStart[k], n = (size_t)(b->particleStart[k + 1] - b->particleStart[k]);
        std::copy(r->pos.begin(), r->pos.end(), pos.begin() + 3 * p0);
        if (!r->vel.empty()) std::copy(r->vel.begin(), r->vel.end(), vel.begin() + 3 * p0);
        if (!r->mass.empty()) std::copy(r->mass.begin(), r->mass.begin() + n, mass.begin() + p0);
        steps[k] = r->steps;
    }
    IX_TRY(batchMdSetup(b, mass.data(), vel.data(), steps.data()));
    return batchCopyIn(b, b->dPos, pos.data(), pos.size() * sizeof(double));
}

int enqueueCohortRun(ServerShard* H, ServerUnit* u) {
    ix_batch* b = u->batch;
    const int nm = (int)u->members.size(), np = b->numParticles;
    IX_BCUDA(b, cudaGraphLaunch(b->graph, b->stream));
    double* st = reinterpret_cast<double*>(u->staging);
    const size_t n3 = 3 * (size_t)np;
    int first = 0;
    for (int step = 0; first < nm; step++) {
        if (step > 0) IX_TRY(batchMdStep(b, u->members[0]->dt));
        int last = first;
        while (last < nm && u->members[last]->steps == step) last++;
        if (last == first) continue;
        const size_t a = 3 * (size_t)b->particleStart[first], e = 3 * (size_t)b->particleStart[last];
        IX_BCUDA(b, cudaMemcpyAsync(st + a, b->dPos + a, (e - a) * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        IX_BCUDA(b, cudaMemcpyAsync(st + n3 + a, b->dVel + a, (e - a) * sizeof(double), cudaMemcpyDeviceToHost,
                                    b->stream));
        IX_BCUDA(b, cudaMemcpyAsync(st + 2 * n3 + a, b->dForces + a, (e - a) * sizeof(double), cudaMemcpyDeviceToHost,
                                    b->stream));
        IX_BCUDA(b, cudaMemcpyAsync(st + 3 * n3 + 4 * (size_t)first, b->dEnergies + 4 * (size_t)first,
                                    4 * (size_t)(last - first) * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        ServerUnit::Mark mk;
        mk.event = shardEvent(H);
        mk.first = first;
        mk.last = last;
        IX_BCUDA(b, cudaEventRecord(mk.event, b->stream));
        u->marks.push_back(mk);
        first = last;
    }
    return IX_OK;
}

// Launch an admitted cohort of small requests (their estimates already reserved) as one batch in the server's arena.
void launchCohort(ix_server* S, ServerShard* H, std::vector<ServerRequest*>& members, size_t reserved) {
    std::stable_sort(members.begin(), members.end(),
                     [](const ServerRequest* a, const ServerRequest* b) { return a->steps < b->steps; });
    ServerUnit* u = new ServerUnit();
    u->members = members;
    u->reserved = reserved;
    ix_batch* b = new ix_batch();
    b->device = S->device;
    b->numSMs = S->numSMs;
    b->arena = &S->arena;
    b->particleStart.push_back(0);
    u->batch = b;
    int rc = IX_OK;
    if (!H->cohortStreams.empty()) {
        b->stream = H->cohortStreams.back();
        H->cohortStreams.pop_back();
    }
    else if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = batchFail(b, IX_ERR_CUDA, "cudaStreamCreate failed");
    for (ServerRequest* r : members) {
        b->systems.push_back(r->sys);   // the batch owns the descriptions from here on
        b->particleStart.push_back(b->particleStart.back() + r->sys->n);
        r->sys = nullptr;
    }
    {
        PhaseTimer t(H->workerSec[2]);
        // the build's uploads go out asynchronously from the unit's pinned staging, after its results area
        b->deferUploads = true;
        if (rc == IX_OK) rc = buildBatch(b);
        if (rc == IX_OK) rc = stageCohortState(u);
        if (rc == IX_OK) {
            const size_t np = (size_t)b->numParticles;
            const size_t results = (9 * np + 4 * members.size()) * sizeof(double);
            u->staging = S->pinned.alloc(results + b->pendingBytes.size());
            if (!u->staging) rc = batchFail(b, IX_ERR_MEMORY, "pinned host staging could not be allocated");
            else rc = flushBatchUploads(b, u->staging + results);
        }
        b->deferUploads = false;
    }
    if (rc == IX_OK) {
        PhaseTimer t(H->workerSec[3]);
        rc = enqueueCohortRun(H, u);
    }
    if (rc != IX_OK) {
        const std::string msg = b->error;
        if (b->stream) cudaStreamSynchronize(b->stream);
        for (auto& mk : u->marks) H->freeEvents.push_back(mk.event);
        if (u->staging) S->pinned.release(u->staging);
        ix_batch_destroy(b);
        unreserveBytes(S, u->reserved);
        for (ServerRequest* r : members) serverFinish(S, H, r, rc, msg);
        delete u;
        return;
    }
    const size_t actual = bufferBytes(b->buffers);
    if (actual > u->reserved) {
        S->reserved += (long long)(actual - u->reserved);
        u->reserved = actual;
    }
    H->units.push_back(u);
    std::lock_guard<std::mutex> lock(S->m);
    S->stats.cohorts++;
    S->stats.admitted += (long long)members.size();
}

// Unpack the members of a finished mark of a cohort from the unit's pinned staging.
void unpackCohortMark(ix_server* S, ServerShard* H, ServerUnit* u, const ServerUnit::Mark& mk) {
    const double* st = reinterpret_cast<const double*>(u->staging);
    const ix_batch* b = u->batch;
    const size_t n3 = 3 * (size_t)b->numParticles;
    for (int k = mk.first; k < mk.last; k++) {
        ServerRequest* r = u->members[k];
        const size_t a = 3 * (size_t)b->particleStart[k], e = 3 * (size_t)b->particleStart[k + 1];
        r->pos.assign(st + a, st + e);
        r->vel.assign(st + n3 + a, st + n3 + e);
        r->forces.assign(st + 2 * n3 + a, st + 2 * n3 + e);
        std::memcpy(r->energies, st + 3 * n3 + 4 * (size_t)k, sizeof(r->energies));
        serverFinish(S, H, r, IX_OK, "");
    }
}

// Release a unit whose requests are all finished (or failed).  A context whose request succeeded goes to the shard's
// pool, keeping its memory reserved, for the next request of the same System.
void releaseUnit(ix_server* S, ServerShard* H, ServerUnit* u, bool succeeded = false) {
    for (auto& mk : u->marks) H->freeEvents.push_back(mk.event);
    u->marks.clear();
    if (u->staging) S->pinned.release(u->staging);
    u->staging = nullptr;
    if (u->ctx) {
        ServerRequest* r = u->members[0];
        r->sys = nullptr;
        if (succeeded && S->maxPooled > 0 && !r->desc.empty()) {
            ix_ctx* c = u->ctx;
            c->uploadBuf = nullptr;          // the staging went back to the pinned pool
            c->uploadCap = c->uploadUsed = 0;
            const size_t actual = bufferBytes(c->buffers);
            if (actual > u->reserved) {
                S->reserved += (long long)(actual - u->reserved);
                u->reserved = actual;
            }
            PooledContext p;
            p.ctx = c;
            p.desc = std::move(r->desc);
            p.reserved = u->reserved;
            p.lastUse = serverNow();
            H->poolBytes += p.reserved;
            H->pool.emplace(r->key, std::move(p));
            u->ctx = nullptr;
            u->reserved = 0;
            while (H->pool.size() > S->maxPooled) evictPooled(S, H);
        }
        else {
            retireContext(S, H, u->ctx);
            u->ctx = nullptr;
        }
    }
    if (u->batch) {
        cudaStreamSynchronize(u->batch->stream);
        H->cohortStreams.push_back(u->batch->stream);   // the stream goes back to the pool
        u->batch->stream = nullptr;
        ix_batch_destroy(u->batch);   // frees the cohort's memory and descriptions
        u->batch = nullptr;
    }
    unreserveBytes(S, u->reserved);
}

// Check the shard's events; finish the requests whose results have arrived.  Returns whether anything finished.
bool collect(ix_server* S, ServerShard* H) {
    bool progress = false;
    for (size_t i = 0; i < H->units.size();) {
        ServerUnit* u = H->units[i];
        int failCode = IX_OK;
        std::string msg;
        while (u->next < u->marks.size()) {
            const ServerUnit::Mark& mk = u->marks[u->next];
            const cudaError_t q = cudaEventQuery(mk.event);
            if (q == cudaErrorNotReady) break;
            progress = true;
            if (q != cudaSuccess) {
                failCode = IX_ERR_CUDA;
                msg = std::string("CUDA error while running the request: ") + cudaGetErrorString(q);
                break;
            }
            if (u->ctx) {
                // an overflow of a neighbor list during the steps: grow the lists and run the request again
                const double* st = reinterpret_cast<const double*>(u->staging);
                const size_t n3 = 3 * (size_t)u->ctx->n;
                int flags[8];
                std::memcpy(flags, st + 3 * n3 + 4, sizeof(flags));
                if (flags[1] || flags[5]) {
                    // a pair-list overflow: grow the list and run the request again; a three-body list overflow
                    // needs no rerun (those sites were scanned in full), the list only grows
                    bool redo = false;
                    int rc = checkOverflow(u->ctx, selectedTerms(u->ctx, -1), redo);
                    if (rc == IX_OK && redo && ++u->restarts <= 3) {
                        H->freeEvents.push_back(mk.event);
                        u->marks.clear();
                        u->ctx->uploadUsed = 0;   // the stream has run every earlier upload
                        rc = enqueueContextRun(H, u);
                        if (rc == IX_OK) continue;
                    }
                    if (rc != IX_OK || redo) {
                        failCode = rc != IX_OK ? rc : IX_ERR_STATE;
                        msg = rc != IX_OK ? u->ctx->error : "neighbor lists kept overflowing";
                        break;
                    }
                }
                ServerRequest* r = u->members[0];
                r->pos.assign(st, st + n3);
                r->vel.assign(st + n3, st + 2 * n3);
                r->forces.assign(st + 2 * n3, st + 3 * n3);
                std::memcpy(r->energies, st + 3 * n3, sizeof(r->energies));
            }
            else unpackCohortMark(S, H, u, u->marks[u->next]);
            u->next++;
        }
        const bool finished = failCode != IX_OK || u->next >= u->marks.size();
        if (!finished) {
            i++;
            continue;
        }
        {
            PhaseTimer t(H->workerSec[4]);
            // the requests not yet finished: a context's one request, or the cohort members from the current mark
            std::vector<ServerRequest*> rest;
            if (u->ctx) rest.push_back(u->members[0]);
            else if (failCode != IX_OK)
                for (size_t m = (size_t)u->marks[u->next].first; m < u->members.size(); m++)
                    rest.push_back(u->members[m]);
            releaseUnit(S, H, u, failCode == IX_OK);
            for (ServerRequest* r : rest) serverFinish(S, H, r, failCode, msg);
        }
        delete u;
        H->units[i] = H->units.back();
        H->units.pop_back();
    }
    return progress;
}

// Admit the shard's pending requests while its running count and the budget allow.  Small requests gather into one
// cohort per pass, which starts when it is full, when its oldest request has waited the batching window, or when the
// shard has nothing else on the GPU; otherwise its requests go back to the queue to wait for more.  A request older
// than a quarter second that does not fit stops the requests behind it from passing it.  Returns whether anything
// was launched.
bool admit(ix_server* S, ServerShard* H) {
    const double now = serverNow();
    std::vector<ServerRequest*> cohort;
    size_t cohortBytes = 0;
    bool launched = false;
    int scanned = 0;
    for (auto it = H->pending.begin(); it != H->pending.end() && scanned < 4096; scanned++) {
        ServerRequest* r = *it;
        if (H->running >= S->maxRunning) break;
        if ((double)r->estimate > S->budget) {
            it = H->pending.erase(it);
            H->running++;
            char buf[160];
            snprintf(buf, sizeof(buf), "the request needs about %zu bytes of device memory; the budget is %.0f",
                     r->estimate, S->budget);
            serverFinish(S, H, r, IX_ERR_MEMORY, buf);
            continue;
        }
        bool taken = false;
        if (r->small) {
            const bool joins = cohort.empty() || ((int)cohort.size() < S->maxCohort && cohortCompatible(r, cohort[0]));
            if (joins && reserveBytes(S, r->estimate)) {
                cohort.push_back(r);
                cohortBytes += r->estimate;
                taken = true;
            }
            else if (!joins) {
                ++it;
                continue;
            }
        }
        else {
            bool fits = hasPooled(H, r);
            if (fits) fits = reserveBytes(S, 0);
            else {
                fits = reserveBytes(S, r->estimate);
                while (!fits && evictPooled(S, H)) fits = reserveBytes(S, r->estimate);
            }
            if (fits) {
                if (hasPooled(H, r)) r->estimate = 0;   // launchContext releases nothing for it
                it = H->pending.erase(it);
                H->running++;
                launchContext(S, H, r);
                launched = true;
                continue;
            }
        }
        if (taken) {
            H->running++;
            it = H->pending.erase(it);
            continue;
        }
        if (now - r->tSubmit > 0.25) break;   // it does not fit: no passing a request that has waited long
        ++it;
    }
    if (!cohort.empty()) {
        const bool full = (int)cohort.size() >= S->maxCohort;
        const bool waited = now - cohort[0]->tSubmit >= S->window;
        if (full || waited || H->units.empty()) {
            launchCohort(S, H, cohort, cohortBytes);
            launched = true;
        }
        else {
            unreserveBytes(S, cohortBytes);
            for (auto r = cohort.rbegin(); r != cohort.rend(); ++r) H->pending.push_front(*r);
            H->running -= (long long)cohort.size();
        }
    }
    return launched;
}

void shardLoop(ix_server* S, ServerShard* H) {
    cudaSetDevice(S->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(S->m);
            if (H->units.empty() && H->pending.empty())
                S->cvSubmit.wait(lock, [&] { return S->stop || !H->incoming.empty(); });
            if (S->stop) break;
            while (!H->incoming.empty()) {
                H->pending.push_back(H->incoming.front());
                H->incoming.pop_front();
            }
        }
        const double l0 = H->workerSec[0] + H->workerSec[1] + H->workerSec[2] + H->workerSec[3];
        const double c0 = H->workerSec[4];
        const double t0 = serverNow();
        const bool admitted = admit(S, H);
        const double t1 = serverNow();
        const bool collected = collect(S, H);
        const double t2 = serverNow();
        H->workerSec[6] += (t1 - t0) - (H->workerSec[0] + H->workerSec[1] + H->workerSec[2] + H->workerSec[3] - l0);
        H->workerSec[5] += (t2 - t1) - (H->workerSec[4] - c0);
        if (!admitted && !collected) {
            PhaseTimer t(H->workerSec[7]);
            std::unique_lock<std::mutex> lock(S->m);
            S->cvSubmit.wait_for(lock, std::chrono::microseconds(20), [&] { return S->stop || !H->incoming.empty(); });
        }
    }
    // shutdown: wait for the units in flight, release them, fail what never ran
    for (ServerUnit* u : H->units) {
        std::vector<ServerRequest*> rest;
        if (u->ctx) {
            cudaStreamSynchronize(u->ctx->stream);
            rest.push_back(u->members[0]);
        }
        else {
            cudaStreamSynchronize(u->batch->stream);
            for (size_t m = u->next < u->marks.size() ? (size_t)u->marks[u->next].first : u->members.size();
                 m < u->members.size(); m++)
                rest.push_back(u->members[m]);
        }
        releaseUnit(S, H, u);
        for (ServerRequest* r : rest) serverFinish(S, H, r, IX_ERR_STATE, "the server was destroyed");
        delete u;
    }
    H->units.clear();
    while (evictPooled(S, H)) {
    }
    for (ServerRequest* r : H->pending) serverFinish(S, nullptr, r, IX_ERR_STATE, "the server was destroyed");
    H->pending.clear();
    for (const StreamSet& set : H->streams) {
        cudaStreamDestroy(set.stream);
        cudaStreamDestroy(set.stream2);
        cudaStreamDestroy(set.body);
        cudaEventDestroy(set.fork);
        cudaEventDestroy(set.join);
    }
    H->streams.clear();
    for (cudaStream_t st : H->cohortStreams) cudaStreamDestroy(st);
    H->cohortStreams.clear();
    for (cudaEvent_t e : H->freeEvents) cudaEventDestroy(e);
    H->freeEvents.clear();
}

int serverFail(ix_server* S, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (S) {
        std::lock_guard<std::mutex> lock(S->m);
        S->error = buf;
    }
    else g_createError = buf;
    return code;
}

}  // namespace

extern "C" {

int ix_request_create(int num_particles, const double* box, ix_ctx** out) {
    if (!out) return fail(nullptr, IX_ERR_INVALID, "ix_request_create: out is NULL");
    *out = nullptr;
    if (num_particles <= 0) return fail(nullptr, IX_ERR_INVALID, "ix_request_create: the System has no particles");
    ix_ctx* c = new ix_ctx();
    c->n = num_particles;
    c->device = -1;
    if (box) {
        std::memcpy(c->defaultBox, box, sizeof(c->defaultBox));
        std::memcpy(c->box, box, sizeof(c->box));
    }
    *out = c;
    return IX_OK;
}

int ix_request_set_state(ix_ctx* request, const double* positions, const double* velocities, const double* masses) {
    if (!request) return IX_ERR_INVALID;
    if (request->stream) return fail(request, IX_ERR_INVALID, "ix_request_set_state: not a request description");
    if (!positions) return fail(request, IX_ERR_INVALID, "ix_request_set_state: positions is NULL");
    const size_t n3 = 3 * (size_t)request->n;
    for (size_t i = 0; i < n3; i++)
        if (!std::isfinite(positions[i]))
            return fail(request, IX_ERR_INVALID, "Particle coordinate is NaN or infinite (particle %zu)", i / 3);
    if (masses)
        for (int i = 0; i < request->n; i++)
            if (!(masses[i] >= 0)) return fail(request, IX_ERR_INVALID, "Illegal mass for particle %d", i);
    request->requestPos.assign(positions, positions + n3);
    if (velocities) request->requestVel.assign(velocities, velocities + n3);
    else request->requestVel.clear();
    if (masses) request->requestMass.assign(masses, masses + request->n);
    else request->requestMass.clear();
    return IX_OK;
}

int ix_server_create(int device, double budget_bytes, int max_running, int threads, ix_server** out) {
    if (!out) return serverFail(nullptr, IX_ERR_INVALID, "ix_server_create: out is NULL");
    *out = nullptr;
    if (!(budget_bytes > 0)) return serverFail(nullptr, IX_ERR_INVALID, "ix_server_create: the budget must be positive");
    if (max_running <= 0) return serverFail(nullptr, IX_ERR_INVALID, "ix_server_create: max_running must be positive");
    if (threads <= 0 || threads > 64)
        return serverFail(nullptr, IX_ERR_INVALID, "ix_server_create: threads must be in 1..64");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return serverFail(nullptr, IX_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= count)
        return serverFail(nullptr, IX_ERR_NO_DEVICE, "CUDA device %d does not exist (%d devices)", device, count);
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major < 10)
        return serverFail(nullptr, IX_ERR_NO_DEVICE, "device %d (sm_%d) is not a Blackwell (sm_100) GPU", device, major);
    ix_server* S = new ix_server();
    S->device = device;
    cudaDeviceGetAttribute(&S->numSMs, cudaDevAttrMultiProcessorCount, device);
    S->budget = budget_bytes;
    S->maxRunning = std::max(1, max_running / threads);
    // the arena's first chunk (up to 4 GB) and the pinned staging are allocated now, before anything runs: growing
    // either while the GPU is busy waits for the device
    S->arena.limit = (size_t)budget_bytes;
    S->arena.chunkBytes = std::min<size_t>(size_t(1) << 30, std::max<size_t>((size_t)budget_bytes / 4, 1 << 20));
    cudaSetDevice(device);
    S->arena.grow(std::min<size_t>((size_t)budget_bytes, size_t(4) << 30));
    S->stats.budget_bytes = budget_bytes;
    S->pinned.chunkBytes = size_t(1) << 30;
    S->pinned.release(S->pinned.alloc(1));
    S->reaper = std::thread(reaperLoop, S);
    // streams and events for every request a shard can run at once, created now: creating them while the GPU is
    // busy waits for it
    for (int k = 0; k < threads; k++) {
        S->shards.emplace_back(new ServerShard());
        ServerShard* H = S->shards.back().get();
        H->index = k;
        cudaSetDevice(device);
        for (int i = 0; i < S->maxRunning; i++) {
            StreamSet set;
            if (cudaStreamCreateWithFlags(&set.stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaStreamCreateWithFlags(&set.stream2, cudaStreamNonBlocking) != cudaSuccess ||
                cudaStreamCreateWithFlags(&set.body, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&set.fork, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&set.join, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                break;
            }
            H->streams.push_back(set);
        }
        for (int i = 0; i < 2 * S->maxRunning; i++) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                break;
            }
            H->freeEvents.push_back(e);
        }
    }
    for (auto& H : S->shards) H->worker = std::thread(shardLoop, S, H.get());
    *out = S;
    return IX_OK;
}

int ix_server_set_batching(ix_server* S, int small_atoms, int max_cohort, double window_seconds) {
    if (!S) return IX_ERR_INVALID;
    if (small_atoms < 0 || max_cohort <= 0 || !(window_seconds >= 0))
        return serverFail(S, IX_ERR_INVALID, "ix_server_set_batching: illegal settings");
    std::lock_guard<std::mutex> lock(S->m);
    S->smallAtoms = small_atoms;
    S->maxCohort = max_cohort;
    S->window = window_seconds;
    return IX_OK;
}

void ix_server_destroy(ix_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lock(S->m);
        S->stop = true;
    }
    S->cvSubmit.notify_all();
    for (auto& H : S->shards)
        if (H->worker.joinable()) H->worker.join();
    {
        std::lock_guard<std::mutex> lock(S->graveM);
        S->graveStop = true;
    }
    S->graveCv.notify_all();
    if (S->reaper.joinable()) S->reaper.join();
    cudaSetDevice(S->device);
    for (auto& H : S->shards)
        for (ServerRequest* r : H->incoming) {
            if (r->sys) ix_ctx_destroy(r->sys);
            delete r;
        }
    for (auto& kv : S->done) delete kv.second;
    delete S;
}

const char* ix_server_last_error(const ix_server* S) { return S ? S->error.c_str() : g_createError.c_str(); }

int ix_server_submit(ix_server* S, ix_ctx* request, int steps, double dt, long long* id) {
    NvtxRange nvtxRange("ix_server_submit");
    if (!S || !request) return IX_ERR_INVALID;
    if (request->stream || request->device != -1)
        return serverFail(S, IX_ERR_INVALID, "ix_server_submit: not a request description (use ix_request_create)");
    if (request->requestPos.size() != 3 * (size_t)request->n)
        return serverFail(S, IX_ERR_STATE, "ix_server_submit: the request's positions have not been set");
    if (steps < 0) return serverFail(S, IX_ERR_INVALID, "ix_server_submit: negative number of steps");
    if (steps > 0 && !(dt > 0)) return serverFail(S, IX_ERR_INVALID, "ix_server_submit: the step size must be positive");
    if (steps > 0 && request->requestMass.empty())
        return serverFail(S, IX_ERR_STATE, "ix_server_submit: masses are required for MD steps");
    if (!request->pairShared && !request->atmPresent)
        return serverFail(S, IX_ERR_INVALID, "ix_server_submit: the request has no forces");
    ServerRequest* r = new ServerRequest();
    r->sys = request;
    r->pos.swap(request->requestPos);
    r->vel.swap(request->requestVel);
    r->mass.swap(request->requestMass);
    r->steps = steps;
    r->dt = steps > 0 ? dt : 0.0;
    r->tSubmit = serverNow();
    const bool small = batchable(request) && request->n <= S->smallAtoms;
    if (!small) {
        // serialized on the submitting thread: the key of the shard's context pool
        r->desc = poolDescription(request, r->mass);
        r->key = hashBytes(r->desc);
    }
    {
        std::lock_guard<std::mutex> lock(S->m);
        r->small = small;
        r->estimate = estimateRequestBytes(request, r->small);
        r->id = S->nextId++;
        // small requests gather on shard 0 (larger cohorts); the others go to the shard that pools their System's
        // contexts
        ServerShard* H = r->small ? S->shards[0].get() : S->shards[r->key % S->shards.size()].get();
        H->incoming.push_back(r);
        S->stats.submitted++;
        if (id) *id = r->id;
    }
    S->cvSubmit.notify_all();
    return IX_OK;
}

static int takeDone(ix_server* S, int max_ids, long long* ids, int* count) {
    int k = 0;
    while (k < max_ids && !S->doneIds.empty()) {
        ids[k++] = S->doneIds.front();
        S->doneIds.pop_front();
    }
    *count = k;
    return IX_OK;
}

int ix_server_poll(ix_server* S, int max_ids, long long* ids, int* count) {
    if (!S || !count || (max_ids > 0 && !ids)) return IX_ERR_INVALID;
    std::lock_guard<std::mutex> lock(S->m);
    return takeDone(S, max_ids, ids, count);
}

int ix_server_wait(ix_server* S, double timeout_seconds, int max_ids, long long* ids, int* count) {
    if (!S || !count || (max_ids > 0 && !ids)) return IX_ERR_INVALID;
    std::unique_lock<std::mutex> lock(S->m);
    S->cvDone.wait_for(lock, std::chrono::duration<double>(std::max(timeout_seconds, 0.0)),
                       [&] { return !S->doneIds.empty(); });
    return takeDone(S, max_ids, ids, count);
}

int ix_server_result(ix_server* S, long long id, double* positions, double* velocities, double* forces,
                     double* term_energies, double* latency_seconds) {
    if (!S) return IX_ERR_INVALID;
    ServerRequest* r = nullptr;
    {
        std::lock_guard<std::mutex> lock(S->m);
        auto it = S->done.find(id);
        if (it == S->done.end()) {
            S->error = "ix_server_result: no completed request with this id";
            return IX_ERR_STATE;
        }
        r = it->second;
        S->done.erase(it);
        if (r->status != IX_OK) S->error = r->error;
    }
    const int status = r->status;
    if (status == IX_OK) {
        if (positions) std::copy(r->pos.begin(), r->pos.end(), positions);
        if (velocities) std::copy(r->vel.begin(), r->vel.end(), velocities);
        if (forces) std::copy(r->forces.begin(), r->forces.end(), forces);
        if (term_energies) std::memcpy(term_energies, r->energies, sizeof(r->energies));
    }
    if (latency_seconds) *latency_seconds = r->tDone - r->tSubmit;
    delete r;
    return status;
}

int ix_server_stats_get(ix_server* S, ix_server_stats* stats) {
    if (!S || !stats) return IX_ERR_INVALID;
    std::lock_guard<std::mutex> lock(S->m);
    *stats = S->stats;
    stats->pending = 0;
    stats->running = 0;
    for (int k = 0; k < 12; k++) stats->worker_seconds[k] = 0;
    for (auto& H : S->shards) {
        stats->pending += (long long)(H->incoming.size() + H->pending.size());
        stats->running += H->running;
        for (int k = 0; k < 12; k++) stats->worker_seconds[k] += H->workerSec[k];
    }
    stats->reserved_bytes = (double)S->reserved.load();
    stats->peak_reserved_bytes = (double)S->peakReserved.load();
    {
        std::lock_guard<std::mutex> alock(S->arena.m);
        stats->arena_bytes = (double)S->arena.inUse;
        stats->peak_arena_bytes = (double)S->arena.peak;
    }
    return IX_OK;
}

}  // extern "C"
