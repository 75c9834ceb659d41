// A request server: continuous batching of independent energy+force / MD requests of mixed sizes on one GPU.
// Included at the end of ix_context.cu (after ix_batch.cuh), whose contexts and batches it runs.
//
// One native worker thread owns the device side.  Each pass of its loop
//   1. moves newly submitted requests into the pending queue (FIFO),
//   2. admits pending requests while the running count and the device memory budget allow (a request whose estimate
//      does not fit waits; later, smaller requests may pass it), launching each admitted periodic request as a
//      context on its own streams and gathering admitted small non-periodic requests into a cohort (an ix_batch run
//      with per-system step counts, one CUDA graph per MD step of the whole cohort),
//   3. checks the events that mark finished requests: their results were copied by their own stream into pinned
//      staging, so the worker only unpacks them, and frees the unit's memory when its last request is done.
// All launches are asynchronous, so every admitted request's work overlaps on the device.  A request's state
// (positions, velocities, parameters, neighbor lists) stays resident on the device from admission to its last step.
// Its results are those of the same request run alone: a context runs the same kernels either way, and a batched
// system's evaluation is independent of the other systems of its batch.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

namespace {

double serverNow() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Host memory that the device can copy into asynchronously: chunks from cudaHostAlloc, sub-allocated first-fit.
struct PinnedPool {
    struct Chunk {
        char* base = nullptr;
        size_t bytes = 0;
        std::map<size_t, size_t> free;
    };
    std::vector<Chunk> chunks;
    std::map<char*, std::pair<size_t, size_t>> live;
    size_t chunkBytes = size_t(64) << 20;

    char* alloc(size_t bytes) {
        bytes = (std::max<size_t>(bytes, 1) + 255) / 256 * 256;
        for (size_t c = 0;; c++) {
            if (c == chunks.size()) {
                Chunk k;
                k.bytes = std::max(chunkBytes, bytes);
                if (cudaHostAlloc(reinterpret_cast<void**>(&k.base), k.bytes, cudaHostAllocDefault) != cudaSuccess) {
                    cudaGetLastError();
                    return nullptr;
                }
                k.free[0] = k.bytes;
                chunks.push_back(std::move(k));
            }
            auto& fr = chunks[c].free;
            for (auto it = fr.begin(); it != fr.end(); ++it) {
                if (it->second < bytes) continue;
                const size_t off = it->first, rest = it->second - bytes;
                fr.erase(it);
                if (rest) fr[off + bytes] = rest;
                char* p = chunks[c].base + off;
                live[p] = {c, bytes};
                return p;
            }
        }
    }

    void release(char* p) {
        auto it = live.find(p);
        if (it == live.end()) return;
        Chunk& k = chunks[it->second.first];
        size_t off = static_cast<size_t>(p - k.base), bytes = it->second.second;
        live.erase(it);
        auto next = k.free.lower_bound(off);
        if (next != k.free.end() && next->first == off + bytes) {
            bytes += next->second;
            next = k.free.erase(next);
        }
        if (next != k.free.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += bytes;
                return;
            }
        }
        k.free[off] = bytes;
    }

    ~PinnedPool() {
        for (auto& k : chunks) cudaFreeHost(k.base);
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
    size_t reserved = 0;                 // device bytes the unit holds
    int restarts = 0;
};

}  // namespace

struct ix_server {
    int device = 0;
    DeviceArena arena;
    PinnedPool pinned;
    double budget = 0.0;
    int maxRunning = 256;
    int smallAtoms = 1024;
    int maxCohort = 512;
    double window = 200e-6;
    std::thread worker;
    std::mutex m;                        // guards incoming, done, doneIds, results, error, stats, stop
    std::condition_variable cvSubmit, cvDone;
    bool stop = false;
    std::deque<ServerRequest*> incoming;
    std::map<long long, ServerRequest*> done;
    std::deque<long long> doneIds;
    long long nextId = 1;
    std::string error;
    ix_server_stats stats{};
    // worker-owned
    std::deque<ServerRequest*> pending;
    std::vector<ServerUnit*> units;
    std::vector<cudaEvent_t> freeEvents;
    size_t reserved = 0;
    long long running = 0;
};

namespace {

// Device bytes a request will hold, an upper bound used for admission (the unit's actual bytes replace it once it
// is launched).  A periodic context holds per-particle arrays, the pair tiles (a few hundred bytes per tile, ~75 tiles
// per 32-particle block at water density and a 1 nm cutoff, with the list's growth margin) and the three-body site
// lists; a batched system holds its all-pairs block tiles and all-sites lists.
size_t estimateRequestBytes(const ix_ctx* c, bool small) {
    const size_t n = (size_t)c->n, sites = c->siteParams.size() / 3, nb = (n + 31) / 32;
    if (small) return (size_t(64) << 10) + 1024 * n + 640 * (nb * (nb + 1) / 2) + 16 * sites * sites + 512 * sites;
    return (size_t(8) << 20) + 6144 * n + 4096 * sites;
}

cudaEvent_t serverEvent(ix_server* S) {
    if (!S->freeEvents.empty()) {
        cudaEvent_t e = S->freeEvents.back();
        S->freeEvents.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
}

void serverFinish(ix_server* S, ServerRequest* r, int status, const std::string& error) {
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
    S->running--;
    S->cvDone.notify_all();
}

// Enqueue a periodic request's whole run on its context's stream: positions, masses and velocities in, the first
// evaluation and every step, then the final state copied into the pinned staging, and the event that marks it done.
int enqueueContextRun(ix_server* S, ServerUnit* u) {
    ServerRequest* r = u->members[0];
    ix_ctx* c = u->ctx;
    const size_t n3 = 3 * (size_t)c->n;
    IX_TRY(ix_set_positions(c, r->pos.data(), nullptr));
    if (r->mass.empty()) r->mass.assign(c->n, 1.0);
    IX_TRY(ix_md_set_masses(c, r->mass.data()));
    if (r->vel.empty()) IX_CUDA(c, cudaMemsetAsync(c->dVel, 0, n3 * sizeof(double), c->stream));
    else IX_CUDA(c, cudaMemcpyAsync(c->dVel, r->vel.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    c->mdForcesValid = false;
    IX_TRY(ix_md_steps_async(c, r->steps, r->dt));
    double* st = reinterpret_cast<double*>(u->staging);
    IX_CUDA(c, cudaMemcpyAsync(st, c->dPos, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    IX_CUDA(c, cudaMemcpyAsync(st + n3, c->dVel, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    IX_CUDA(c, cudaMemcpyAsync(st + 2 * n3, c->dOutForces, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    IX_CUDA(c, cudaMemcpyAsync(st + 3 * n3, c->dOutEnergy, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    IX_CUDA(c, cudaMemcpyAsync(st + 3 * n3 + 4, c->dFlags, 8 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ServerUnit::Mark mk;
    mk.event = serverEvent(S);
    mk.first = 0;
    mk.last = 1;
    IX_CUDA(c, cudaEventRecord(mk.event, c->stream));
    u->marks.assign(1, mk);
    u->next = 0;
    return IX_OK;
}

// Admit a periodic request: its description becomes a device context in the server's arena.
void launchContext(ix_server* S, ServerRequest* r) {
    ServerUnit* u = new ServerUnit();
    u->members.push_back(r);
    ix_ctx* c = r->sys;
    c->arena = &S->arena;
    c->device = S->device;
    u->ctx = c;
    size_t before;
    {
        std::lock_guard<std::mutex> lock(S->arena.m);
        before = S->arena.inUse;
    }
    int rc = ctxInitDevice(c);
    if (rc == IX_OK) {
        u->staging = S->pinned.alloc((9 * (size_t)c->n + 8) * sizeof(double));
        if (!u->staging) rc = fail(c, IX_ERR_MEMORY, "pinned host staging could not be allocated");
    }
    if (rc == IX_OK) rc = enqueueContextRun(S, u);
    {
        std::lock_guard<std::mutex> lock(S->arena.m);
        u->reserved = S->arena.inUse - before;
    }
    if (rc != IX_OK) {
        const std::string msg = c->error;
        if (c->stream) cudaStreamSynchronize(c->stream);
        for (auto& mk : u->marks) S->freeEvents.push_back(mk.event);
        if (u->staging) S->pinned.release(u->staging);
        u->ctx = nullptr;
        delete u;
        serverFinish(S, r, rc, msg);   // destroys the context and frees its memory
        return;
    }
    S->reserved += u->reserved;
    S->units.push_back(u);
    std::lock_guard<std::mutex> lock(S->m);
    S->stats.contexts++;
    S->stats.admitted++;
}

// Whether a small request can join a cohort started by c0: the same force settings, parameters and step size.
bool cohortCompatible(const ServerRequest* r, const ServerRequest* r0) {
    return r->dt == r0->dt && r->sys->parameters == r0->sys->parameters && sameBatchSettings(r->sys, r0->sys);
}

// Enqueue a cohort's whole run on its batch's stream: the first evaluation, then every step up to the longest
// request; after the last step of each group of requests (members are ordered by steps) their final state is copied
// into the pinned staging and an event marks them done.
int enqueueCohortRun(ix_server* S, ServerUnit* u) {
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
    IX_BCUDA(b, cudaMemcpyAsync(b->dPos, pos.data(), pos.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    IX_BCUDA(b, cudaStreamSynchronize(b->stream));   // the host vectors go out of scope
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
        mk.event = serverEvent(S);
        mk.first = first;
        mk.last = last;
        IX_BCUDA(b, cudaEventRecord(mk.event, b->stream));
        u->marks.push_back(mk);
        first = last;
    }
    return IX_OK;
}

// Admit a cohort of small requests as one batch in the server's arena.
void launchCohort(ix_server* S, std::vector<ServerRequest*>& members) {
    std::stable_sort(members.begin(), members.end(),
                     [](const ServerRequest* a, const ServerRequest* b) { return a->steps < b->steps; });
    ServerUnit* u = new ServerUnit();
    u->members = members;
    ix_batch* b = new ix_batch();
    b->device = S->device;
    b->arena = &S->arena;
    b->particleStart.push_back(0);
    u->batch = b;
    size_t before;
    {
        std::lock_guard<std::mutex> lock(S->arena.m);
        before = S->arena.inUse;
    }
    int rc = IX_OK;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, S->device) == cudaSuccess) b->numSMs = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = batchFail(b, IX_ERR_CUDA, "cudaStreamCreate failed");
    for (ServerRequest* r : members) {
        b->systems.push_back(r->sys);   // the batch owns the descriptions from here on
        b->particleStart.push_back(b->particleStart.back() + r->sys->n);
        r->sys = nullptr;
    }
    if (rc == IX_OK) rc = buildBatch(b);
    if (rc == IX_OK) {
        const size_t np = (size_t)b->numParticles;
        u->staging = S->pinned.alloc((9 * np + 4 * members.size()) * sizeof(double));
        if (!u->staging) rc = batchFail(b, IX_ERR_MEMORY, "pinned host staging could not be allocated");
    }
    if (rc == IX_OK) rc = enqueueCohortRun(S, u);
    {
        std::lock_guard<std::mutex> lock(S->arena.m);
        u->reserved = S->arena.inUse - before;
    }
    if (rc != IX_OK) {
        const std::string msg = b->error;
        if (b->stream) cudaStreamSynchronize(b->stream);
        for (auto& mk : u->marks) S->freeEvents.push_back(mk.event);
        if (u->staging) S->pinned.release(u->staging);
        ix_batch_destroy(b);
        for (ServerRequest* r : members) serverFinish(S, r, rc, msg);
        delete u;
        return;
    }
    S->reserved += u->reserved;
    S->units.push_back(u);
    std::lock_guard<std::mutex> lock(S->m);
    S->stats.cohorts++;
    S->stats.admitted += (long long)members.size();
}

// Unpack the members of a finished mark from the unit's pinned staging.
void unpackMark(ix_server* S, ServerUnit* u, const ServerUnit::Mark& mk) {
    const double* st = reinterpret_cast<const double*>(u->staging);
    if (u->ctx) {
        ServerRequest* r = u->members[0];
        const size_t n3 = 3 * (size_t)u->ctx->n;
        r->pos.assign(st, st + n3);
        r->vel.assign(st + n3, st + 2 * n3);
        r->forces.assign(st + 2 * n3, st + 3 * n3);
        std::memcpy(r->energies, st + 3 * n3, sizeof(r->energies));
        return;
    }
    const ix_batch* b = u->batch;
    const size_t n3 = 3 * (size_t)b->numParticles;
    for (int k = mk.first; k < mk.last; k++) {
        ServerRequest* r = u->members[k];
        const size_t a = 3 * (size_t)b->particleStart[k], e = 3 * (size_t)b->particleStart[k + 1];
        r->pos.assign(st + a, st + e);
        r->vel.assign(st + n3 + a, st + n3 + e);
        r->forces.assign(st + 2 * n3 + a, st + 2 * n3 + e);
        std::memcpy(r->energies, st + 3 * n3 + 4 * (size_t)k, sizeof(r->energies));
        serverFinish(S, r, IX_OK, "");
    }
}

void releaseUnit(ix_server* S, ServerUnit* u) {
    for (auto& mk : u->marks) S->freeEvents.push_back(mk.event);
    u->marks.clear();
    if (u->staging) S->pinned.release(u->staging);
    u->staging = nullptr;
    if (u->batch) ix_batch_destroy(u->batch);   // frees the cohort's memory and descriptions
    u->batch = nullptr;
    S->reserved -= u->reserved;
}

// Check the units' events; finish the requests whose results have arrived.  Returns whether anything finished.
bool collect(ix_server* S) {
    bool progress = false;
    for (size_t i = 0; i < S->units.size();) {
        ServerUnit* u = S->units[i];
        bool failed = false;
        std::string msg;
        while (u->next < u->marks.size()) {
            const ServerUnit::Mark& mk = u->marks[u->next];
            const cudaError_t q = cudaEventQuery(mk.event);
            if (q == cudaErrorNotReady) break;
            progress = true;
            if (q != cudaSuccess) {
                failed = true;
                msg = std::string("CUDA error while running the request: ") + cudaGetErrorString(q);
                break;
            }
            if (u->ctx) {
                // an overflow of a neighbor list during the steps: grow the lists and run the request again
                int flags[8];
                std::memcpy(flags, reinterpret_cast<const double*>(u->staging) + 9 * (size_t)u->ctx->n + 4,
                            sizeof(flags));
                if (flags[1] || flags[5]) {
                    bool redo = false;
                    int rc = checkOverflow(u->ctx, selectedTerms(u->ctx, -1), redo);
                    if (rc == IX_OK && ++u->restarts <= 3) {
                        S->freeEvents.push_back(mk.event);
                        u->marks.clear();
                        rc = enqueueContextRun(S, u);
                        if (rc == IX_OK) continue;
                    }
                    failed = true;
                    msg = rc != IX_OK ? u->ctx->error : "neighbor lists kept overflowing";
                    break;
                }
            }
            unpackMark(S, u, mk);
            u->next++;
        }
        if (failed) {
            if (u->ctx) {
                ServerRequest* r = u->members[0];
                cudaStreamSynchronize(u->ctx->stream);
                r->sys = nullptr;
                releaseUnit(S, u);
                ix_ctx_destroy(u->ctx);
                u->ctx = nullptr;
                serverFinish(S, r, IX_ERR_CUDA, msg);
            }
            else {
                cudaStreamSynchronize(u->batch->stream);
                for (size_t m = (size_t)u->marks[u->next].first; m < u->members.size(); m++)
                    serverFinish(S, u->members[m], IX_ERR_CUDA, msg);
                releaseUnit(S, u);
            }
            delete u;
            S->units[i] = S->units.back();
            S->units.pop_back();
            continue;
        }
        if (u->next >= u->marks.size()) {
            if (u->ctx) {
                ServerRequest* r = u->members[0];
                r->sys = nullptr;
                releaseUnit(S, u);
                ix_ctx_destroy(u->ctx);   // frees the context's memory in the arena
                u->ctx = nullptr;
                serverFinish(S, r, IX_OK, "");
            }
            else releaseUnit(S, u);
            delete u;
            S->units[i] = S->units.back();
            S->units.pop_back();
            continue;
        }
        i++;
    }
    return progress;
}

// Admit pending requests while the running count and the budget allow.  Small requests gather into one cohort per
// pass, which starts when it is full, when its oldest request has waited the batching window, or when the GPU has
// nothing else to do; otherwise its requests go back to the queue to wait for more.  A request older than a quarter
// second that does not fit stops the requests behind it from passing it.  Returns whether anything was launched.
bool admit(ix_server* S) {
    const double now = serverNow();
    const double budget = S->budget;
    std::vector<ServerRequest*> cohort;
    size_t cohortBytes = 0;
    bool launched = false;
    int scanned = 0;
    for (auto it = S->pending.begin(); it != S->pending.end() && scanned < 4096; scanned++) {
        ServerRequest* r = *it;
        if (S->running >= S->maxRunning) break;
        if ((double)r->estimate > budget) {
            it = S->pending.erase(it);
            S->running++;
            char buf[160];
            snprintf(buf, sizeof(buf), "the request needs about %zu bytes of device memory; the budget is %.0f",
                     r->estimate, budget);
            serverFinish(S, r, IX_ERR_MEMORY, buf);
            continue;
        }
        const bool fits = (double)(S->reserved + cohortBytes + r->estimate) <= budget;
        if (r->small) {
            const bool joins = cohort.empty() || ((int)cohort.size() < S->maxCohort && cohortCompatible(r, cohort[0]));
            if (joins && fits) {
                cohort.push_back(r);
                cohortBytes += r->estimate;
                S->running++;
                it = S->pending.erase(it);
                continue;
            }
        }
        else if (fits) {
            it = S->pending.erase(it);
            S->running++;
            launchContext(S, r);
            launched = true;
            continue;
        }
        if (!fits && now - r->tSubmit > 0.25) break;   // no passing a request that has waited long
        ++it;
    }
    if (!cohort.empty()) {
        const bool full = (int)cohort.size() >= S->maxCohort;
        const bool waited = now - cohort[0]->tSubmit >= S->window;
        if (full || waited || S->units.empty()) {
            launchCohort(S, cohort);
            launched = true;
        }
        else {
            for (auto r = cohort.rbegin(); r != cohort.rend(); ++r) S->pending.push_front(*r);
            S->running -= (long long)cohort.size();
        }
    }
    return launched;
}

void serverLoop(ix_server* S) {
    cudaSetDevice(S->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(S->m);
            if (S->units.empty() && S->pending.empty())
                S->cvSubmit.wait(lock, [&] { return S->stop || !S->incoming.empty(); });
            if (S->stop) break;
            while (!S->incoming.empty()) {
                S->pending.push_back(S->incoming.front());
                S->incoming.pop_front();
            }
        }
        const bool progress = admit(S) | collect(S);
        {
            std::lock_guard<std::mutex> lock(S->m);
            S->stats.pending = (long long)S->pending.size() + (long long)S->incoming.size();
            S->stats.running = S->running;
            S->stats.reserved_bytes = (double)S->reserved;
            S->stats.peak_reserved_bytes = std::max(S->stats.peak_reserved_bytes, (double)S->reserved);
        }
        if (!progress) {
            std::unique_lock<std::mutex> lock(S->m);
            S->cvSubmit.wait_for(lock, std::chrono::microseconds(20), [&] { return S->stop || !S->incoming.empty(); });
        }
    }
    // shutdown: wait for the units in flight, release them, fail what never ran
    for (ServerUnit* u : S->units) {
        if (u->ctx) {
            cudaStreamSynchronize(u->ctx->stream);
            u->members[0]->sys = nullptr;
            releaseUnit(S, u);
            ix_ctx_destroy(u->ctx);
            u->ctx = nullptr;
            serverFinish(S, u->members[0], IX_ERR_STATE, "the server was destroyed");
        }
        else {
            cudaStreamSynchronize(u->batch->stream);
            for (size_t m = u->next < u->marks.size() ? (size_t)u->marks[u->next].first : u->members.size();
                 m < u->members.size(); m++)
                serverFinish(S, u->members[m], IX_ERR_STATE, "the server was destroyed");
            releaseUnit(S, u);
        }
        delete u;
    }
    S->units.clear();
    for (ServerRequest* r : S->pending) serverFinish(S, r, IX_ERR_STATE, "the server was destroyed");
    S->pending.clear();
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

int ix_server_create(int device, double budget_bytes, int max_running, ix_server** out) {
    if (!out) return serverFail(nullptr, IX_ERR_INVALID, "ix_server_create: out is NULL");
    *out = nullptr;
    if (!(budget_bytes > 0)) return serverFail(nullptr, IX_ERR_INVALID, "ix_server_create: the budget must be positive");
    if (max_running <= 0) return serverFail(nullptr, IX_ERR_INVALID, "ix_server_create: max_running must be positive");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return serverFail(nullptr, IX_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= count)
        return serverFail(nullptr, IX_ERR_NO_DEVICE, "CUDA device %d does not exist (%d devices)", device, count);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    if (prop.major < 10)
        return serverFail(nullptr, IX_ERR_NO_DEVICE, "device %d (%s, sm_%d%d) is not a Blackwell (sm_100) GPU", device,
                          prop.name, prop.major, prop.minor);
    ix_server* S = new ix_server();
    S->device = device;
    S->budget = budget_bytes;
    S->maxRunning = max_running;
    S->arena.limit = (size_t)budget_bytes;
    S->arena.chunkBytes = std::min<size_t>(S->arena.chunkBytes, std::max<size_t>((size_t)budget_bytes / 4, 1 << 20));
    S->stats.budget_bytes = budget_bytes;
    S->worker = std::thread(serverLoop, S);
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
    if (S->worker.joinable()) S->worker.join();
    cudaSetDevice(S->device);
    for (ServerRequest* r : S->incoming) {
        if (r->sys) ix_ctx_destroy(r->sys);
        delete r;
    }
    for (auto& kv : S->done) delete kv.second;
    for (cudaEvent_t e : S->freeEvents) cudaEventDestroy(e);
    delete S;
}

const char* ix_server_last_error(const ix_server* S) { return S ? S->error.c_str() : g_createError.c_str(); }

int ix_server_submit(ix_server* S, ix_ctx* request, int steps, double dt, long long* id) {
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
    {
        std::lock_guard<std::mutex> lock(S->m);
        r->small = batchable(request) && request->n <= S->smallAtoms;
        r->estimate = estimateRequestBytes(request, r->small);
        r->id = S->nextId++;
        S->incoming.push_back(r);
        S->stats.submitted++;
        if (id) *id = r->id;
    }
    S->cvSubmit.notify_one();
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
    {
        std::lock_guard<std::mutex> alock(S->arena.m);
        stats->arena_bytes = (double)S->arena.inUse;
        stats->peak_arena_bytes = (double)S->arena.peak;
    }
    return IX_OK;
}

}  // extern "C"
