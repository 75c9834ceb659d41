// Restatement of the reference's CPU platform for the short-range path: the timed CPU baseline of bench.py.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY (like the rest of oracle/): it is never part of the product path.
//
// What the reference's CPU platform does, restated here in portable C++ threads:
//   * each pair force is its own pass (CpuInteraxPairForceFvec.h:136-394, one object per force in
//     CpuInteraxKernels.cpp:77-219) in single precision: positions in float, the pair terms of InteraxPairTerms.h
//     evaluated in float (here the templated terms of interax_oracle.hpp at T = float), forces summed per thread in
//     float and energies in double;
//   * its neighbor list (OpenMM's CpuNeighborList) is rebuilt for every evaluation: the particles are sorted into
//     voxels and cut into blocks of 8 consecutive sorted particles; each block lists the particles that may be
//     within the cutoff of any of its members; threads take blocks from an atomic counter, one lane per block member;
//   * the three-body force (CpuInteraxThreeBodyForce.cpp:39-188) in double precision: site centroids and an
//     all-pairs neighbor search split over the threads, then the triples by marking (a site C is a neighbor of A and
//     of B < C when it carries A's mark and appears in B's list), sites taken from an atomic counter, per-thread site
//     forces combined at the end.
// Like the reference with AVX (fvec8, CpuInteraxPairForceAvx.cpp:44-48), each block of eight is evaluated against
// each listed neighbor with one eight-lane vector (cpu_simd.h): the block's particles in the lanes, the neighbor
// broadcast, exclusions as a per-neighbor lane mask built with the list.
#include "interax_oracle.hpp"
#include "cpu_simd.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>

namespace ixo {
namespace {

// A persistent pool of host threads: run(f) calls f(thread index) on every thread and waits (OpenMM's ThreadPool
// plays this part on the reference's CPU platform).
class ThreadPool {
public:
    explicit ThreadPool(int n) : count(n) {
        for (int i = 1; i < n; i++) workers.emplace_back([this, i] { loop(i); });
    }
    ~ThreadPool() {
        {
            std::lock_guard<std::mutex> lock(m);
            stop = true;
            generation++;
        }
        cv.notify_all();
        for (auto& t : workers) t.join();
    }
    int size() const { return count; }
    void run(const std::function<void(int)>& f) {
        {
            std::lock_guard<std::mutex> lock(m);
            task = &f;
            pending = count - 1;
            generation++;
        }
        cv.notify_all();
        f(0);
        std::unique_lock<std::mutex> lock(m);
        done.wait(lock, [&] { return pending == 0; });
        task = nullptr;
    }

private:
    void loop(int index) {
        unsigned long long seen = 0;
        for (;;) {
            const std::function<void(int)>* f;
            {
                std::unique_lock<std::mutex> lock(m);
                cv.wait(lock, [&] { return generation != seen; });
                seen = generation;
                if (stop) return;
                f = task;
            }
            (*f)(index);
            std::lock_guard<std::mutex> lock(m);
            if (--pending == 0) done.notify_all();
        }
    }
    int count;
    std::vector<std::thread> workers;
    std::mutex m;
    std::condition_variable cv, done;
    const std::function<void(int)>* task = nullptr;
    int pending = 0;
    unsigned long long generation = 0;
    bool stop = false;
};

ThreadPool& pool(int threads) {
    static std::unique_ptr<ThreadPool> p;
    if (!p || p->size() != threads) {
        p.reset();
        p.reset(new ThreadPool(threads));
    }
    return *p;
}

constexpr int kBlock = 8;

struct Float3 {
    float x, y, z;
};

// Minimum image of a float displacement in a reduced box (c, then b, then a), as the CPU platform applies it.
inline void minimumImage(float& dx, float& dy, float& dz, const float box[3][3], const float invDiag[3],
                         bool triclinic) {
    if (!triclinic) {
        dx -= box[0][0] * std::nearbyint(dx * invDiag[0]);
        dy -= box[1][1] * std::nearbyint(dy * invDiag[1]);
        dz -= box[2][2] * std::nearbyint(dz * invDiag[2]);
        return;
    }
    float s = std::floor(dz * invDiag[2] + 0.5f);
    dx -= s * box[2][0];
    dy -= s * box[2][1];
    dz -= s * box[2][2];
    s = std::floor(dy * invDiag[1] + 0.5f);
    dx -= s * box[1][0];
    dy -= s * box[1][1];
    s = std::floor(dx * invDiag[0] + 0.5f);
    dx -= s * box[0][0];
}

// One pair force as the CPU platform holds it after initialize(): float parameters, exclusion sets, the long-range
// correction coefficients.
struct CpuPairForce {
    PairTerm term;
    int n = 0, stride = 0;
    PairSettings settings;
    std::vector<float> params;              // n x stride
    std::vector<uint8_t> alch;
    std::vector<std::vector<int>> excl;     // sorted partners of each particle
    float dampingScale = 1.0f;
    SlaterTaylorScheme scheme = SlaterTaylorScheme::accurate(true);
    bool anyAlch = false;
    double lrcCoef = 0.0, lrcAlchCoef = 0.0;
    // per evaluation
    std::vector<float> pos;                 // n x 3
    std::vector<int> sorted, sortedPos;
    std::vector<std::vector<int>> blockNbrs;
    std::vector<std::vector<uint8_t>> blockExcl;   // per listed neighbor: the block lanes it is excluded from
    std::vector<std::vector<float>> threadForce;
    std::vector<double> threadEnergy;
    std::vector<long long> threadCount;
};

// The neighbor list of one evaluation: particles sorted into cells of edge >= cutoff, blocks of kBlock consecutive
// sorted particles, and for each block the particles later in the sorted order that may lie within the cutoff of the
// block's bounding box.  Without a cutoff every later particle is listed.
void buildNeighborList(CpuPairForce& F, const float box[3][3], const float invDiag[3], bool periodic, bool triclinic,
                       ThreadPool& tp) {
    const int n = F.n;
    const bool useCutoff = F.settings.method != 0;
    const float cutoff = (float)F.settings.cutoff;
    F.sorted.resize(n);
    F.sortedPos.resize(n);
    const int nb = (n + kBlock - 1) / kBlock;
    F.blockNbrs.assign(nb, {});
    F.blockExcl.assign(nb, {});
    if (!useCutoff) {
        for (int i = 0; i < n; i++) F.sorted[i] = F.sortedPos[i] = i;
        std::atomic<int> next(0);
        tp.run([&](int) {
            std::vector<uint8_t> exclMark(n, 0);
            for (int b = next++; b < nb; b = next++) {
                const int k0 = b * kBlock, k1 = std::min(n, k0 + kBlock);
                for (int k = k0; k < k1; k++)
                    for (int j : F.excl[k]) exclMark[j] |= (uint8_t)(1u << (k - k0));
                auto& list = F.blockNbrs[b];
                for (int j = k0 + 1; j < n; j++) {
                    list.push_back(j);
                    F.blockExcl[b].push_back(exclMark[j]);
                }
                for (int k = k0; k < k1; k++)
                    for (int j : F.excl[k]) exclMark[j] = 0;
            }
        });
        return;
    }
    // cell grid: the periodic box, or the particles' bounding box
    float lo[3], ext[3];
    int nc[3];
    for (int d = 0; d < 3; d++) {
        if (periodic) {
            lo[d] = 0.0f;
            ext[d] = box[d][d];
        }
        else {
            float mn = F.pos[d], mx = F.pos[d];
            for (int i = 1; i < n; i++) {
                mn = std::min(mn, F.pos[3 * i + d]);
                mx = std::max(mx, F.pos[3 * i + d]);
            }
            lo[d] = mn;
            ext[d] = std::max(mx - mn, 1e-6f);
        }
        nc[d] = std::max(1, std::min(1024, (int)(2.0f * ext[d] / cutoff)));   // cells of at least half the cutoff
    }
    const int numCells = nc[0] * nc[1] * nc[2];
    std::vector<int> cellOf(n), cellCount(numCells + 1, 0);
    for (int i = 0; i < n; i++) {
        float f[3] = {F.pos[3 * i], F.pos[3 * i + 1], F.pos[3 * i + 2]};
        if (periodic) {
            // into the reduced cell: c, then b, then a
            float s = std::floor(f[2] * invDiag[2]);
            for (int d = 0; d < 3; d++) f[d] -= s * box[2][d];
            s = std::floor(f[1] * invDiag[1]);
            for (int d = 0; d < 3; d++) f[d] -= s * box[1][d];
            s = std::floor(f[0] * invDiag[0]);
            f[0] -= s * box[0][0];
        }
        int c[3];
        for (int d = 0; d < 3; d++) c[d] = std::min(std::max((int)((f[d] - lo[d]) / ext[d] * nc[d]), 0), nc[d] - 1);
        cellOf[i] = (c[2] * nc[1] + c[1]) * nc[0] + c[0];
        cellCount[cellOf[i] + 1]++;
    }
    for (int c = 0; c < numCells; c++) cellCount[c + 1] += cellCount[c];
    std::vector<int> fill(cellCount.begin(), cellCount.end() - 1);
    for (int i = 0; i < n; i++) F.sorted[fill[cellOf[i]]++] = i;
    for (int k = 0; k < n; k++) F.sortedPos[F.sorted[k]] = k;
    const float cutoff2 = cutoff * cutoff;
    std::atomic<int> next(0);
    tp.run([&](int) {
        std::vector<int> stamp(numCells, -1);
        std::vector<uint8_t> exclMark(n, 0);     // lanes of the current block that exclude each particle
        for (int b = next++; b < nb; b = next++) {
            const int k0 = b * kBlock, k1 = std::min(n, k0 + kBlock);
            for (int k = k0; k < k1; k++)
                for (int j : F.excl[F.sorted[k]]) exclMark[j] |= (uint8_t)(1u << (k - k0));
            // block center and half extents (minimum image from the first member when periodic)
            const int i0 = F.sorted[k0];
            float mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
            for (int k = k0; k < k1; k++) {
                const int i = F.sorted[k];
                float d[3] = {F.pos[3 * i] - F.pos[3 * i0], F.pos[3 * i + 1] - F.pos[3 * i0 + 1],
                              F.pos[3 * i + 2] - F.pos[3 * i0 + 2]};
                if (periodic) minimumImage(d[0], d[1], d[2], box, invDiag, triclinic);
                for (int e = 0; e < 3; e++) {
                    mn[e] = std::min(mn[e], d[e]);
                    mx[e] = std::max(mx[e], d[e]);
                }
            }
            float center[3], half[3];
            for (int e = 0; e < 3; e++) {
                center[e] = F.pos[3 * i0 + e] + 0.5f * (mn[e] + mx[e]);
                half[e] = 0.5f * (mx[e] - mn[e]);
            }
            auto& list = F.blockNbrs[b];
            auto& exclOut = F.blockExcl[b];
            auto scanCell = [&](int cell) {
                if (stamp[cell] == b) return;
                stamp[cell] = b;
                for (int q = std::max(cellCount[cell], k0 + 1); q < cellCount[cell + 1]; q++) {
                    // only particles later in the sorted order
                    const int j = F.sorted[q];
                    if (!triclinic) {
                        // distance from j's nearest image to the block's box (the box is far smaller than half the
                        // periodic box, so the image nearest the center is the nearest to the box)
                        float r2 = 0.0f;
                        for (int e = 0; e < 3; e++) {
                            float d = F.pos[3 * j + e] - center[e];
                            if (periodic) d -= box[e][e] * std::nearbyint(d * invDiag[e]);
                            const float out = std::max(std::fabs(d) - half[e], 0.0f);
                            r2 += out * out;
                        }
                        if (r2 >= cutoff2) continue;
                    }
                    // triclinic: every candidate; the pair loop applies the cutoff
                    list.push_back(j);
                    exclOut.push_back(exclMark[j]);
                }
            };
            if (triclinic) {
                // the images across a tilted face are shifted by whole cells: every cell is a candidate
                for (int c = 0; c < numCells; c++) scanCell(c);
            }
            else {
                // the cells that overlap the block's box grown by the cutoff, per axis (every cell of an axis whose
                // range would wrap onto itself)
                int from[3], count[3];
                for (int e = 0; e < 3; e++) {
                    const float cell = ext[e] / nc[e];
                    const float a = (center[e] - half[e] - cutoff - lo[e]) / cell;
                    const float z = (center[e] + half[e] + cutoff - lo[e]) / cell;
                    from[e] = (int)std::floor(a);
                    count[e] = (int)std::floor(z) - from[e] + 1;
                    if (periodic && count[e] >= nc[e]) {
                        from[e] = 0;
                        count[e] = nc[e];
                    }
                }
                for (int cz = from[2]; cz < from[2] + count[2]; cz++)
                    for (int cy = from[1]; cy < from[1] + count[1]; cy++)
                        for (int cx = from[0]; cx < from[0] + count[0]; cx++) {
                            int x = cx, y = cy, z = cz;
                            if (periodic) {
                                x = ((x % nc[0]) + nc[0]) % nc[0];
                                y = ((y % nc[1]) + nc[1]) % nc[1];
                                z = ((z % nc[2]) + nc[2]) % nc[2];
                            }
                            else if (x < 0 || y < 0 || z < 0 || x >= nc[0] || y >= nc[1] || z >= nc[2])
                                continue;
                            scanCell((z * nc[1] + y) * nc[0] + x);
                        }
            }
            for (int k = k0; k < k1; k++)
                for (int j : F.excl[F.sorted[k]]) exclMark[j] = 0;
        }
    });
}

// One evaluation of a pair force: the neighbor list, then the blocks over the threads.  Energy returned; forces
// added to `forces` (n x 3, double).
double evaluatePairForce(CpuPairForce& F, const double* xyz, const double* box9, double lambda, int threads,
                         double* forces, long long* numInteracting) {
    ThreadPool& tp = pool(threads);
    const int n = F.n, T = tp.size();
    const bool periodic = F.settings.method == 2, useCutoff = F.settings.method != 0;
    float box[3][3] = {{0}}, invDiag[3] = {1, 1, 1};
    bool triclinic = false;
    if (periodic) {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) box[a][b] = (float)box9[3 * a + b];
        for (int d = 0; d < 3; d++) invDiag[d] = (float)(1.0 / box9[4 * d]);
        triclinic = box9[3] != 0 || box9[6] != 0 || box9[7] != 0;
    }
    F.pos.resize(3 * (size_t)n);
    for (size_t k = 0; k < 3 * (size_t)n; k++) F.pos[k] = (float)xyz[k];
    buildNeighborList(F, box, invDiag, periodic, triclinic, tp);
    if (!F.anyAlch) lambda = 1.0;
    const float lam = (float)lambda;
    const float cutoff = (float)F.settings.cutoff, cutoff2 = cutoff * cutoff;
    const bool useSwitch = useCutoff && F.settings.useSwitch;
    const float sw = (float)F.settings.switchDistance, invSwitchWidth = useSwitch ? 1.0f / (cutoff - sw) : 0.0f;
    const float soft6 = F.settings.softcoreRadius > 0 ? (float)std::pow(F.settings.softcoreRadius, 6.0) : 0.0f;
    F.threadForce.resize(T);
    F.threadEnergy.assign(T, 0.0);
    F.threadCount.assign(T, 0);
    const int nb = (n + kBlock - 1) / kBlock, st = F.stride;
    const bool orderByIndex = !F.scheme.aboutSmallerWidth;
    std::atomic<int> next(0);
    tp.run([&](int t) {
        using namespace simd;
        std::vector<float>& fo = F.threadForce[t];
        fo.assign(3 * (size_t)n, 0.0f);
        double energy = 0.0;
        long long count = 0;
        const V8 cut2(cutoff2);
        for (int b = next++; b < nb; b = next++) {
            const int k0 = b * kBlock, k1 = std::min(n, k0 + kBlock);
            // the block's particles, one lane each (padding lanes repeat the last particle and stay masked)
            float bx[kBlock], by[kBlock], bz[kBlock], bi[kBlock], ba[kBlock], bp[5][kBlock];
            for (int l = 0; l < kBlock; l++) {
                const int i = F.sorted[std::min(k0 + l, k1 - 1)];
                bx[l] = F.pos[3 * i];
                by[l] = F.pos[3 * i + 1];
                bz[l] = F.pos[3 * i + 2];
                bi[l] = (float)i;
                ba[l] = (float)F.alch[i];
                for (int k = 0; k < st; k++) bp[k][l] = F.params[(size_t)i * st + k];
            }
            const V8 X = V8::load(bx), Y = V8::load(by), Z = V8::load(bz), I = V8::load(bi), AL = V8::load(ba);
            V8 P[5];
            for (int k = 0; k < st; k++) P[k] = V8::load(bp[k]);
            V8 fX, fY, fZ, eBlock;
            const unsigned valid = (1u << (k1 - k0)) - 1u;
            const std::vector<int>& list = F.blockNbrs[b];
            const std::vector<uint8_t>& exclBits = F.blockExcl[b];
            for (size_t q = 0; q < list.size(); q++) {
                const int j = list[q];
                const int sj = F.sortedPos[j];
                // lanes before j in the sorted order (each pair once), not excluded
                const unsigned later = sj - k0 >= kBlock ? 0xffu : ((1u << (sj - k0)) - 1u);
                const unsigned lanes = valid & later & ~(unsigned)exclBits[q];
                if (!lanes) continue;
                V8 dx = V8(F.pos[3 * j]) - X, dy = V8(F.pos[3 * j + 1]) - Y, dz = V8(F.pos[3 * j + 2]) - Z;
                if (periodic) {
                    if (triclinic) {
                        V8 s3 = vround(dz * V8(invDiag[2]));
                        dx -= s3 * V8(box[2][0]);
                        dy -= s3 * V8(box[2][1]);
                        dz -= s3 * V8(box[2][2]);
                        V8 s2 = vround(dy * V8(invDiag[1]));
                        dx -= s2 * V8(box[1][0]);
                        dy -= s2 * V8(box[1][1]);
                        dx -= vround(dx * V8(invDiag[0])) * V8(box[0][0]);
                    }
                    else {
                        dx -= vround(dx * V8(invDiag[0])) * V8(box[0][0]);
                        dy -= vround(dy * V8(invDiag[1])) * V8(box[1][1]);
                        dz -= vround(dz * V8(invDiag[2])) * V8(box[2][2]);
                    }
                }
                const V8 r2 = dx * dx + dy * dy + dz * dz;
                V8 include = laneMask(lanes);
                if (useCutoff) include = include & (r2 < cut2);
                const float* pj = &F.params[(size_t)j * st];
                V8 Q[5];
                for (int k = 0; k < st; k++) Q[k] = V8(pj[k]);
                const int gate = F.term == kDispersion ? 3 : (F.term == kExchange ? 1 : 2);
                include = include & (P[gate] * Q[gate] > V8(0.0f));
                if (!any(include)) continue;
                const V8 r = vsqrt(r2);
                const V8 alchLane = vabs(AL - V8((float)F.alch[j])) > V8(0.5f);
                V8 rEff = r, softFactor(1.0f);
                if (soft6 > 0 && any(alchLane & include)) {
                    // per lane, as the reference does for the soft-core distance
                    float rv[kBlock], av[kBlock], re[kBlock], fa[kBlock];
                    r.store(rv);
                    select(alchLane, V8(1.0f), V8(0.0f)).store(av);
                    for (int l = 0; l < kBlock; l++) {
                        re[l] = av[l] != 0 ? std::pow(rv[l] * rv[l] * rv[l] * rv[l] * rv[l] * rv[l] + (1.0f - lam) *
                                                      soft6, 1.0f / 6.0f) : rv[l];
                        const float qr = rv[l] / re[l];
                        fa[l] = av[l] != 0 ? qr * qr * qr * qr * qr : 1.0f;
                    }
                    rEff = V8::load(re);
                    softFactor = V8::load(fa);
                }
                // the order-2 overlap expands about the width of the particle with the lower index: it goes first
                V8 A[5], C[5];
                const V8 blockFirst = I < V8((float)j);
                for (int k = 0; k < st; k++) {
                    A[k] = orderByIndex ? select(blockFirst, P[k], Q[k]) : P[k];
                    C[k] = orderByIndex ? select(blockFirst, Q[k], P[k]) : Q[k];
                }
                V8 e, dEdR;
                if (F.term == kDispersion) dispersionPair(rEff, A, C, F.dampingScale, e, dEdR);
                else if (F.term == kExchange) exchangePair(rEff, A, C, F.scheme, e, dEdR);
                else shortRangePair(rEff, A, C, F.scheme, e, dEdR);
                dEdR *= softFactor;
                if (useSwitch) {
                    const V8 u = zeroUnless(r > V8(sw), (r - V8(sw)) * V8(invSwitchWidth));
                    const V8 sv = V8(1.0f) + u * u * u * (V8(-10.0f) + u * (V8(15.0f) - u * V8(6.0f)));
                    const V8 sd = u * u * (V8(-30.0f) + u * (V8(60.0f) - u * V8(30.0f))) * V8(invSwitchWidth);
                    dEdR = dEdR * sv + e * sd;
                    e *= sv;
                }
                const V8 scale = select(alchLane, V8(lam), V8(1.0f));
                eBlock += zeroUnless(include, scale * e);
                // force on the block particle i: dE/dr (x_j - x_i)/r
                const V8 fs = zeroUnless(include, scale * dEdR / r);
                const V8 fx = dx * fs, fy = dy * fs, fz = dz * fs;
                fX += fx;
                fY += fy;
                fZ += fz;
                fo[3 * j] -= sum(fx);
                fo[3 * j + 1] -= sum(fy);
                fo[3 * j + 2] -= sum(fz);
                count += __builtin_popcount((unsigned)_mm256_movemask_ps(include.v));
            }
            energy += (double)sum(eBlock);
            float ox[kBlock], oy[kBlock], oz[kBlock];
            fX.store(ox);
            fY.store(oy);
            fZ.store(oz);
            for (int k = k0; k < k1; k++) {
                const int i = F.sorted[k];
                fo[3 * i] += ox[k - k0];
                fo[3 * i + 1] += oy[k - k0];
                fo[3 * i + 2] += oz[k - k0];
            }
        }
        F.threadEnergy[t] = energy;
        F.threadCount[t] = count;
    });
    // the per-thread forces into the output, split over the threads by particle
    tp.run([&](int t) {
        for (int i = t; i < n; i += T)
            for (int d = 0; d < 3; d++) {
                double sum = 0.0;
                for (int u = 0; u < T; u++) sum += F.threadForce[u][3 * (size_t)i + d];
                forces[3 * (size_t)i + d] += sum;
            }
    });
    double energy = 0.0;
    long long count = 0;
    for (int t = 0; t < T; t++) {
        energy += F.threadEnergy[t];
        count += F.threadCount[t];
    }
    if (F.term == kDispersion && periodic && (F.lrcCoef != 0 || F.lrcAlchCoef != 0))
        energy += (F.lrcCoef + lambda * F.lrcAlchCoef) / (box9[0] * box9[4] * box9[8]);
    if (numInteracting) *numInteracting = count;
    return energy;
}

// The three-body force as the CPU platform holds it (CpuInteraxThreeBodyForce.cpp:39-78).
struct CpuThreeBody {
    ThreeBodySettings s;
    std::vector<int> molecule;
    std::vector<Vec3> sites;
    std::vector<std::vector<int>> nbr;
    std::vector<std::vector<Vec3>> threadSiteForce;
    std::vector<std::vector<int>> threadMarks;
    std::vector<double> threadEnergy;
    std::vector<long long> threadCount;
};

double evaluateThreeBody(CpuThreeBody& A, const double* xyz, const double* box9, double lambda, int threads,
                         double* forces, long long* numTriples) {
    ThreadPool& tp = pool(threads);
    const ThreeBodySettings& s = A.s;
    const int ns = (int)s.siteParticles.size(), T = tp.size();
    Vec3 box[3];
    for (int k = 0; k < 3; k++) box[k] = Vec3(box9[3 * k], box9[3 * k + 1], box9[3 * k + 2]);
    bool anyAlch = false;
    for (auto a : s.alch) anyAlch |= (a != 0);
    if (!anyAlch) lambda = 1.0;
    A.sites.resize(ns);
    A.nbr.resize(ns);
    A.threadSiteForce.resize(T);
    A.threadMarks.resize(T);
    A.threadEnergy.assign(T, 0.0);
    A.threadCount.assign(T, 0);
    auto delta = [&](const Vec3& from, const Vec3& to) { return s.periodic ? periodicDelta(from, to, box) : to - from; };
    // site centroids, split over the threads
    tp.run([&](int t) {
        for (int i = t; i < ns; i += T) {
            Vec3 c;
            for (int p : s.siteParticles[i]) c += Vec3(xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2]);
            A.sites[i] = c / double(s.siteParticles[i].size());
        }
    });
    // neighbors B > A of other molecules within the cutoff: all pairs, split over the threads
    const double cutoff2 = s.cutoff * s.cutoff;
    tp.run([&](int t) {
        for (int i = t; i < ns; i += T) {
            std::vector<int>& list = A.nbr[i];
            list.clear();
            for (int j = i + 1; j < ns; j++) {
                if (A.molecule[i] == A.molecule[j]) continue;
                const Vec3 d = delta(A.sites[i], A.sites[j]);
                if (d.dot(d) < cutoff2) list.push_back(j);
            }
        }
    });
    // triples by marking, sites A from a counter
    const bool useDamping = s.dampingMethod == 1;
    std::atomic<int> next(0);
    tp.run([&](int t) {
        std::vector<Vec3>& sf = A.threadSiteForce[t];
        sf.assign(ns, Vec3());
        std::vector<int>& marks = A.threadMarks[t];
        marks.assign(ns, -1);
        double energy = 0.0;
        long long count = 0;
        for (int a = next++; a < ns; a = next++) {
            for (int b : A.nbr[a]) marks[b] = a;
            for (int b : A.nbr[a])
                for (int c : A.nbr[b]) {
                    if (marks[c] != a) continue;
                    double c9 = s.scale * atmC9(s.alpha[a], s.frequency[a], s.alpha[b], s.frequency[b], s.alpha[c],
                                                s.frequency[c]);
                    if (s.alch[a] || s.alch[b] || s.alch[c]) c9 *= lambda;
                    if (c9 == 0) continue;
                    const double rates[3] = {2 * s.dampingScale / (s.width[a] + s.width[b]),
                                             2 * s.dampingScale / (s.width[a] + s.width[c]),
                                             2 * s.dampingScale / (s.width[b] + s.width[c])};
                    energy += atmTriple(delta(A.sites[a], A.sites[b]), delta(A.sites[a], A.sites[c]),
                                        delta(A.sites[b], A.sites[c]), c9, useDamping ? rates : nullptr, sf[a], sf[b],
                                        sf[c], s.centroidRadius);
                    count++;
                }
        }
        A.threadEnergy[t] = energy;
        A.threadCount[t] = count;
    });
    // site forces shared among each site's particles
    for (int i = 0; i < ns; i++) {
        Vec3 f;
        for (int t = 0; t < T; t++) f += A.threadSiteForce[t][i];
        f = f / double(s.siteParticles[i].size());
        for (int p : s.siteParticles[i]) {
            forces[3 * p] += f.x;
            forces[3 * p + 1] += f.y;
            forces[3 * p + 2] += f.z;
        }
    }
    double energy = 0.0;
    long long count = 0;
    for (int t = 0; t < T; t++) {
        energy += A.threadEnergy[t];
        count += A.threadCount[t];
    }
    if (numTriples) *numTriples = count;
    return energy;
}

}  // namespace
}  // namespace ixo

// ----------------------------------------------------------------------------------------------------------------------
// C interface for ctypes: create (the CPU kernels' initialize()), evaluate (execute()), destroy.
// ----------------------------------------------------------------------------------------------------------------------
using namespace ixo;

extern "C" {

int ox_cpu_threads() { return std::max(1u, std::thread::hardware_concurrency()); }

void* ox_cpu_pair_create(int term, int n, const ox_pair_settings* settings, const double* params,
                         const unsigned char* alch, double damping_scale, int use_lrc, int overlap_method) {
    CpuPairForce* F = new CpuPairForce();
    F->term = PairTerm(term);
    F->n = n;
    F->stride = term == 0 ? 5 : (term == 1 ? 2 : 3);
    F->settings.method = settings->method;
    F->settings.cutoff = settings->cutoff;
    F->settings.useSwitch = settings->use_switch != 0;
    F->settings.switchDistance = settings->switch_distance;
    F->settings.softcoreRadius = settings->softcore_radius;
    F->params.resize((size_t)n * F->stride);
    for (size_t k = 0; k < F->params.size(); k++) F->params[k] = (float)params[k];
    F->alch.assign(alch, alch + n);
    for (auto a : F->alch) F->anyAlch |= (a != 0);
    F->excl.assign(n, {});
    for (int e = 0; e < settings->num_exclusions; e++) {
        const int p = settings->exclusions[2 * e], q = settings->exclusions[2 * e + 1];
        F->excl[p].push_back(q);
        F->excl[q].push_back(p);
    }
    for (auto& v : F->excl) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    }
    F->dampingScale = (float)damping_scale;
    // the single-precision switch of the exact method, as the float instantiation of the pair terms uses
    F->scheme = overlap_method == 0 ? SlaterTaylorScheme::accurate(false) : SlaterTaylorScheme::interaxOrder2();
    if (term == 0 && use_lrc && settings->method == 2) {
        PairParams p;
        p.stride = 5;
        p.p.assign(params, params + (size_t)n * 5);
        p.alch.assign(alch, alch + n);
        p.dampingScale = damping_scale;
        p.useLongRangeCorrection = true;
        longRangeCorrection(F->settings, p, F->lrcCoef, F->lrcAlchCoef);
    }
    return F;
}

double ox_cpu_pair_evaluate(void* handle, const double* xyz, const double* box9, double lambda, int threads,
                            double* forces, long long* num_interacting) {
    return evaluatePairForce(*static_cast<CpuPairForce*>(handle), xyz, box9, lambda, std::max(1, threads), forces,
                             num_interacting);
}

void ox_cpu_pair_destroy(void* handle) { delete static_cast<CpuPairForce*>(handle); }

void* ox_cpu_three_body_create(int num_sites, const int* site_offsets, const int* site_particles,
                               const double* site_params, const int* molecule, const unsigned char* alch,
                               double cutoff, double scale, int damping_method, double damping_scale,
                               double centroid_radius, int periodic) {
    CpuThreeBody* A = new CpuThreeBody();
    ThreeBodySettings& s = A->s;
    s.siteParticles.resize(num_sites);
    for (int i = 0; i < num_sites; i++) {
        s.siteParticles[i].assign(site_particles + site_offsets[i], site_particles + site_offsets[i + 1]);
        s.alpha.push_back(site_params[3 * i]);
        s.frequency.push_back(site_params[3 * i + 1]);
        s.width.push_back(site_params[3 * i + 2]);
    }
    s.molecule.assign(molecule, molecule + num_sites);
    s.alch.assign(alch, alch + num_sites);
    s.cutoff = cutoff;
    s.scale = scale;
    s.dampingMethod = damping_method;
    s.dampingScale = damping_scale;
    s.centroidRadius = centroid_radius;
    s.periodic = periodic != 0;
    A->molecule.resize(num_sites);
    for (int i = 0; i < num_sites; i++) A->molecule[i] = molecule[i] < 0 ? -1 - i : molecule[i];
    return A;
}

double ox_cpu_three_body_evaluate(void* handle, const double* xyz, const double* box9, double lambda, int threads,
                                  double* forces, long long* num_triples) {
    return evaluateThreeBody(*static_cast<CpuThreeBody*>(handle), xyz, box9, lambda, std::max(1, threads), forces,
                             num_triples);
}

void ox_cpu_three_body_destroy(void* handle) { delete static_cast<CpuThreeBody*>(handle); }

}  // extern "C"
