// FP64 oracle drivers and their C interface.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, by the smoke check and by bench.py's CPU-baseline leg through ctypes.
// The product never links or loads it.
#include "interax_oracle.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <thread>
#include <set>
#include <unordered_map>

namespace ixo {

// Sum of |pair or triple energies| of the last evaluation on this thread (reset at the start of each one).
static double& lastAbsEnergy() {
    static thread_local double value = 0.0;
    return value;
}

// Threads for a loop of `work` items: every hardware thread for large loops (the split is fixed for a given thread
// count, so the sums are reproducible), one below 100000 items.
static int oracleThreads(size_t work) {
    if (work < 100000) return 1;
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hw ? hw : 1u, 64u));
}

static bool isRectangular(const Vec3* box) {
    return box[1].x == 0 && box[2].x == 0 && box[2].y == 0;
}

void candidatePairs(int n, const std::vector<Vec3>& pos, const Vec3* box, const PairSettings& s,
                    std::vector<std::pair<int, int>>& out) {
    out.clear();
    std::vector<std::vector<int>> excl(n);
    for (auto& e : s.exclusions) {
        excl[e.first].push_back(e.second);
        excl[e.second].push_back(e.first);
    }
    for (auto& v : excl) std::sort(v.begin(), v.end());
    auto excluded = [&](int i, int j) { return std::binary_search(excl[i].begin(), excl[i].end(), j); };
    bool periodic = (s.method == 2);
    bool useCells = (s.method != 0 && n > 2000);
    int nc[3] = {1, 1, 1};
    Vec3 lo, hi;
    if (useCells) {
        if (periodic) {
            if (!isRectangular(box)) useCells = false;
            else {
                double L[3] = {box[0].x, box[1].y, box[2].z};
                for (int k = 0; k < 3; k++) {
                    nc[k] = std::max(1, int(std::floor(L[k] / (s.cutoff * 1.0001))));
                    if (nc[k] < 3) useCells = false;
                }
            }
        }
        else {
            lo = hi = pos[0];
            for (auto& p : pos) {
                lo = Vec3(std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z));
                hi = Vec3(std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z));
            }
            for (int k = 0; k < 3; k++) nc[k] = std::max(1, int(std::floor((hi[k] - lo[k]) / (s.cutoff * 1.0001))));
        }
    }
    if (!useCells) {
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
                if (!excluded(i, j)) out.push_back({i, j});
        return;
    }
    // Cell list: every pair closer than the cutoff lies in the same or adjacent cells.
    auto cellOf = [&](const Vec3& p, int c[3]) {
        for (int k = 0; k < 3; k++) {
            double L = periodic ? (k == 0 ? box[0].x : (k == 1 ? box[1].y : box[2].z)) : (hi[k] - lo[k]);
            double origin = periodic ? 0.0 : lo[k];
            double f = (p[k] - origin) / L;
            if (periodic) f -= std::floor(f);
            int ci = int(f * nc[k]);
            c[k] = std::min(std::max(ci, 0), nc[k] - 1);
        }
    };
    int numCells = nc[0] * nc[1] * nc[2];
    std::vector<std::vector<int>> cells(numCells);
    std::vector<int> cellIndex(n);
    for (int i = 0; i < n; i++) {
        int c[3];
        cellOf(pos[i], c);
        cellIndex[i] = (c[2] * nc[1] + c[1]) * nc[0] + c[0];
        cells[cellIndex[i]].push_back(i);
    }
    // the particles split over threads in contiguous ranges; each range's pairs sorted by (i, j), so the ranges
    // joined in order give the pairs in (i, j) order
    auto range = [&](int first, int last, std::vector<std::pair<int, int>>& dst) {
        std::vector<int> js;
        for (int i = first; i < last; i++) {
            int c[3] = {cellIndex[i] % nc[0], (cellIndex[i] / nc[0]) % nc[1], cellIndex[i] / (nc[0] * nc[1])};
            js.clear();
            for (int dz = -1; dz <= 1; dz++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dx = -1; dx <= 1; dx++) {
                        int cc[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
                        bool skip = false;
                        for (int k = 0; k < 3; k++) {
                            if (periodic) cc[k] = (cc[k] + nc[k]) % nc[k];
                            else if (cc[k] < 0 || cc[k] >= nc[k]) skip = true;
                        }
                        if (skip) continue;
                        for (int j : cells[(cc[2] * nc[1] + cc[1]) * nc[0] + cc[0]])
                            if (j > i && !excluded(i, j)) js.push_back(j);
                    }
            std::sort(js.begin(), js.end());
            js.erase(std::unique(js.begin(), js.end()), js.end());   // small grids visit a cell more than once
            for (int j : js) dst.push_back({i, j});
        }
    };
    const int threads = oracleThreads((size_t)n * 50);
    std::vector<std::vector<std::pair<int, int>>> parts(threads);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
        pool.emplace_back([&, t]() { range((int)((long long)n * t / threads), (int)((long long)n * (t + 1) / threads),
                                           parts[t]); });
    for (auto& th : pool) th.join();
    for (auto& part : parts) out.insert(out.end(), part.begin(), part.end());
}

double computePairForce(PairTerm term, const std::vector<Vec3>& pos, const Vec3* box, const PairSettings& s,
                        const PairParams& params, double lambda, std::vector<Vec3>& forces,
                        int64_t* numInteracting, OpCounter* ops) {
    int n = int(pos.size());
    lastAbsEnergy() = 0.0;
    bool periodic = (s.method == 2);
    bool useCutoff = (s.method != 0);
    bool useSwitch = useCutoff && s.useSwitch;
    bool anyAlch = false;
    for (auto a : params.alch) anyAlch |= (a != 0);
    // The alchemical parameter is read only when some particle is alchemical (ReferenceInteraxKernels.cpp:63-65).
    if (!anyAlch) lambda = 1.0;
    SlaterTaylorScheme scheme = params.overlapMethod == 0 ? SlaterTaylorScheme::accurate(true)
                                                          : SlaterTaylorScheme::interaxOrder2();
    std::vector<std::pair<int, int>> pairs;
    candidatePairs(n, pos, box, s, pairs);
    const int st = params.stride;
    const double* P = params.p.data();
    // one pair; the pair loop is split over threads in fixed contiguous shares (below), each with its own sums
    auto evalPair = [&](const std::pair<int, int>& pr, Vec3* F, double& total, double& absSum, int64_t& count) {
        int i = pr.first, j = pr.second;
        Vec3 d = periodic ? periodicDelta(pos[i], pos[j], box) : pos[j] - pos[i];
        double r = std::sqrt(d.dot(d));
        if (useCutoff && r >= s.cutoff) return;
        bool alchPair = (params.alch[i] != 0) != (params.alch[j] != 0);
        double rEff = r;
        if (alchPair && s.softcoreRadius > 0) {
            double r3 = s.softcoreRadius * s.softcoreRadius * s.softcoreRadius;
            rEff = std::pow(r * r * r * r * r * r + (1 - lambda) * r3 * r3, 1.0 / 6.0);
        }
        double e, dEdR;
        // InteraxOrder2 expands about the width of the particle with the lower index
        // (ReferenceInteraxKernels.cpp:132-134); i < j here.
        const double* a = P + size_t(i) * st;
        const double* b = P + size_t(j) * st;
        if (term == kDispersion) {
            if (a[3] * b[3] == 0) return;
            dispersionPair(rEff, a[0], a[1], a[2], a[3], a[4], b[0], b[1], b[2], b[3], b[4], params.dampingScale, e,
                           dEdR);
        }
        else if (term == kExchange) {
            if (a[1] * b[1] == 0) return;
            exchangePair(rEff, a[0], a[1], b[0], b[1], scheme, e, dEdR);
        }
        else {
            if (a[2] * b[2] == 0) return;
            shortRangePair(rEff, a[0], a[1], a[2], b[0], b[1], b[2], scheme, e, dEdR);
        }
        count++;
        if (ops) {
            // the same term evaluated on counting values
            OpCounter& oc = opCounter();
            oc = OpCounter();
            Counted ce, cd;
            if (term == kDispersion)
                dispersionPair<Counted>(rEff, a[0], a[1], a[2], a[3], a[4], b[0], b[1], b[2], b[3], b[4],
                                        params.dampingScale, ce, cd);
            else if (term == kExchange) exchangePair<Counted>(rEff, a[0], a[1], b[0], b[1], scheme, ce, cd);
            else shortRangePair<Counted>(rEff, a[0], a[1], a[2], b[0], b[1], b[2], scheme, ce, cd);
            ops->arith += oc.arith;
            ops->transcendental += oc.transcendental;
        }
        if (rEff != r) dEdR *= std::pow(r / rEff, 5);
        // sum of |pair energies| before switching: the error scale of tests/TestInteraxPairForce.h:105-142
        absSum += std::fabs((alchPair ? lambda : 1.0) * e);
        if (useSwitch && r > s.switchDistance) {
            double t = (r - s.switchDistance) / (s.cutoff - s.switchDistance);
            double sv = 1 + t * t * t * (-10 + t * (15 - t * 6));
            double sd = t * t * (-30 + t * (60 - t * 30)) / (s.cutoff - s.switchDistance);
            dEdR = dEdR * sv + e * sd;
            e *= sv;
        }
        double scale = alchPair ? lambda : 1.0;
        total += scale * e;
        double fs = scale * dEdR / r;
        Vec3 f(d.x * fs, d.y * fs, d.z * fs);
        F[i] += f;
        F[j] -= f;
    };
    double total = 0, absSum = 0;
    int64_t count = 0;
    const size_t numPairs = pairs.size();
    const int threads = ops ? 1 : oracleThreads(numPairs);
    if (threads <= 1) {
        for (auto& pr : pairs) evalPair(pr, forces.data(), total, absSum, count);
    }
    else {
        std::vector<std::vector<Vec3>> F(threads, std::vector<Vec3>(n));
        std::vector<double> tot(threads, 0.0), abss(threads, 0.0);
        std::vector<int64_t> cnt(threads, 0);
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; t++)
            pool.emplace_back([&, t]() {
                const size_t b = numPairs * t / threads, e = numPairs * (t + 1) / threads;
                for (size_t k = b; k < e; k++) evalPair(pairs[k], F[t].data(), tot[t], abss[t], cnt[t]);
            });
        for (auto& th : pool) th.join();
        for (int t = 0; t < threads; t++) {
            total += tot[t];
            absSum += abss[t];
            count += cnt[t];
            for (int i = 0; i < n; i++) forces[i] += F[t][i];
        }
    }
    lastAbsEnergy() = absSum;
    if (term == kDispersion && params.useLongRangeCorrection && s.method == 2) {
        double coef, alchCoef;
        longRangeCorrection(s, params, coef, alchCoef);
        if (coef != 0 || alchCoef != 0) total += (coef + lambda * alchCoef) / (box[0].x * box[1].y * box[2].z);
    }
    if (numInteracting) *numInteracting = count;
    return total;
}

// Gauss-Legendre rule on (0, 1) by Newton iteration on P_n (InteraxDispersionForceImpl.cpp:49-73).
static void gaussLegendre(int n, std::vector<double>& nodes, std::vector<double>& weights) {
    nodes.resize(n);
    weights.resize(n);
    for (int i = 0; i < n; i++) {
        double x = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1, p1 = x;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (x * p1 - p0) / (x * x - 1);
            double step = p1 / dp;
            x -= step;
            if (std::fabs(step) < 1e-15) break;
        }
        nodes[i] = 0.5 * (1 - x);
        weights[i] = 1 / ((1 - x * x) * dp * dp);
    }
}

void longRangeCorrection(const PairSettings& s, const PairParams& params, double& coefficient,
                         double& alchemicalCoefficient) {
    coefficient = alchemicalCoefficient = 0;
    if (s.method != 2 || !params.useLongRangeCorrection) return;
    typedef std::tuple<double, double, double, double, double, bool> Class;
    std::map<Class, int> counts;
    int n = int(params.alch.size());
    const double* P = params.p.data();
    for (int i = 0; i < n; i++) {
        const double* a = P + size_t(i) * params.stride;
        counts[std::make_tuple(a[0], a[1], a[2], a[3], a[4], params.alch[i] != 0)]++;
    }
    std::vector<std::pair<Class, int>> classes(counts.begin(), counts.end());
    const int numPoints = 32;
    std::vector<double> nodes, weights;
    gaussLegendre(numPoints, nodes, weights);
    double cutoff = s.cutoff;
    double sw = s.useSwitch ? s.switchDistance : cutoff;
    double width = cutoff - sw;
    auto energyAt = [&](double r, const Class& c1, const Class& c2) {
        double e, de;
        dispersionPair(r, std::get<0>(c1), std::get<1>(c1), std::get<2>(c1), std::get<3>(c1), std::get<4>(c1),
                       std::get<0>(c2), std::get<1>(c2), std::get<2>(c2), std::get<3>(c2), std::get<4>(c2),
                       params.dampingScale, e, de);
        return e;
    };
    double sum = 0, alchSum = 0;
    for (size_t i = 0; i < classes.size(); i++)
        for (size_t j = i; j < classes.size(); j++) {
            const Class& c1 = classes[i].first;
            const Class& c2 = classes[j].first;
            if (std::get<3>(c1) * std::get<3>(c2) == 0) continue;
            double integral = 0;
            for (int k = 0; k < numPoints; k++) {
                double u = nodes[k];
                integral += weights[k] * energyAt(cutoff / u, c1, c2) * cutoff * cutoff * cutoff / (u * u * u * u);
                if (s.useSwitch) {
                    double x = nodes[k];
                    double r = sw + x * width;
                    double oneMinusSwitch = x * x * x * (10 + x * (-15 + x * 6));
                    integral += weights[k] * width * oneMinusSwitch * energyAt(r, c1, c2) * r * r;
                }
            }
            double n1 = classes[i].second, n2 = classes[j].second;
            double count = (i == j ? 0.5 * n1 * (n1 + 1) : n1 * n2);
            if (std::get<5>(c1) || std::get<5>(c2)) alchSum += count * integral;
            else sum += count * integral;
        }
    double N = n;
    double norm = 2 * M_PI * N * N / (0.5 * N * (N + 1));
    coefficient = norm * sum;
    alchemicalCoefficient = norm * alchSum;
}

// ------------------------------------------------------------------------------------------------------------------
// ATM
// ------------------------------------------------------------------------------------------------------------------

// Tang-Toennies f_3: InteraxThreeBodyTerms.h:51-65.
template <class T>
static void tangToennies3(T x, T& f, T& df) {
    T e = vexp(-x);
    T t3 = x * x * x / T(6.0);
    df = e * t3;
    if (vval(x) < 2) {
        T term = t3, tail = T(0.0);
        for (int k = 4; k <= 30; k++) {
            term = term * (x / T(double(k)));
            tail = tail + term;
        }
        f = e * tail;
    }
    else f = T(1.0) - e * (T(1.0) + x + x * x / T(2.0) + t3);
}

// g(r) = 1 - exp(-(r/R0)^6): InteraxThreeBodyTerms.h:71-77.
template <class T>
static void centroidDamping(T r, T invR0, T& g, T& dg) {
    T x = r * invR0;
    T x6 = x * x * x;
    x6 = x6 * x6;
    g = T(-std::expm1(-vval(x6)));
    dg = T(6.0) * x6 * vexp(-x6) / r;
}

// One triple: InteraxThreeBodyTerms.h:97-146.  T is double, or the counting type (then the returned forces are
// discarded).
template <class T>
static double computeTripleT(const Vec3& av, const Vec3& bv, const Vec3& cv, double c9d, const double* ratesd,
                             Vec3& fA, Vec3& fB, Vec3& fC, double radius) {
    T a[3] = {T(av.x), T(av.y), T(av.z)}, b[3] = {T(bv.x), T(bv.y), T(bv.z)}, c[3] = {T(cv.x), T(cv.y), T(cv.z)};
    T c9 = T(c9d);
    auto dot = [](const T* x, const T* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
    T u = dot(a, a), v = dot(b, b), w = dot(c, c);
    T p = dot(a, b), q = dot(a, c), s = dot(b, c);
    T invP = T(1.0) / (u * v * w);
    T invP32 = invP * vsqrt(invP);
    T invP52 = invP32 * invP;
    T pqs = p * q * s;
    T energy = c9 * (invP32 - T(3.0) * pqs * invP52);
    T radial = c9 * (T(-3.0) * invP32 + T(15.0) * pqs * invP52);
    T cross = T(-3.0) * c9 * invP52;
    T dEda[3], dEdb[3], dEdc[3];
    for (int k = 0; k < 3; k++) {
        dEda[k] = a[k] * (radial / u) + (b[k] * (q * s) + c[k] * (p * s)) * cross;
        dEdb[k] = b[k] * (radial / v) + (a[k] * (q * s) + c[k] * (p * q)) * cross;
        dEdc[k] = c[k] * (radial / w) + (a[k] * (p * s) + b[k] * (p * q)) * cross;
    }
    if (ratesd != nullptr || radius > 0) {
        T len[3] = {vsqrt(u), vsqrt(v), vsqrt(w)};
        T f[3], dfdr[3];
        for (int i = 0; i < 3; i++) {
            if (ratesd != nullptr) {
                T rate = T(ratesd[i]);
                tangToennies3<T>(rate * len[i], f[i], dfdr[i]);
                dfdr[i] = dfdr[i] * rate;
            }
            else {
                f[i] = T(1.0);
                dfdr[i] = T(0.0);
            }
            if (radius > 0) {
                T g, dg;
                centroidDamping<T>(len[i], T(1.0) / T(radius), g, dg);
                dfdr[i] = dfdr[i] * g + f[i] * dg;
                f[i] = f[i] * g;
            }
        }
        T damping = f[0] * f[1] * f[2];
        T sa = energy * dfdr[0] * f[1] * f[2] / len[0];
        T sb = energy * f[0] * dfdr[1] * f[2] / len[1];
        T sc = energy * f[0] * f[1] * dfdr[2] / len[2];
        for (int k = 0; k < 3; k++) {
            dEda[k] = dEda[k] * damping + a[k] * sa;
            dEdb[k] = dEdb[k] * damping + b[k] * sb;
            dEdc[k] = dEdc[k] * damping + c[k] * sc;
        }
        energy = energy * damping;
    }
    Vec3 ga(vval(dEda[0]), vval(dEda[1]), vval(dEda[2]));
    Vec3 gb(vval(dEdb[0]), vval(dEdb[1]), vval(dEdb[2]));
    Vec3 gc(vval(dEdc[0]), vval(dEdc[1]), vval(dEdc[2]));
    fA += ga + gb;
    fB += gc - ga;
    fC -= gb + gc;
    return vval(energy);
}

static double computeC9(double a1, double w1, double a2, double w2, double a3, double w3) {
    return 1.5 * a1 * a2 * a3 * w1 * w2 * w3 * (w1 + w2 + w3) / ((w1 + w2) * (w2 + w3) * (w3 + w1));
}

double atmTriple(const Vec3& ab, const Vec3& ac, const Vec3& bc, double c9, const double* rates, Vec3& fA, Vec3& fB,
                 Vec3& fC, double centroidRadius) {
    return computeTripleT<double>(ab, ac, bc, c9, rates, fA, fB, fC, centroidRadius);
}

double atmC9(double a1, double w1, double a2, double w2, double a3, double w3) {
    return computeC9(a1, w1, a2, w2, a3, w3);
}

// ReferenceInteraxThreeBodyIxn::calculateIxn (ReferenceInteraxThreeBodyIxn.cpp:84-135).  The reference builds an
// N x N neighbor matrix and loops over i < j < k; here each site keeps the sorted list of its neighbors above it and
// the triples are enumerated in the same i, j, k order, so the energies and forces are summed in the same order.
double computeThreeBody(const std::vector<Vec3>& pos, const Vec3* box, const ThreeBodySettings& s, double lambda,
                        std::vector<Vec3>& forces, int64_t* numTriples, OpCounter* ops) {
    int ns = int(s.siteParticles.size());
    lastAbsEnergy() = 0.0;
    bool anyAlch = false;
    for (auto a : s.alch) anyAlch |= (a != 0);
    if (!anyAlch) lambda = 1.0;
    std::vector<int> molecule(ns);
    for (int i = 0; i < ns; i++) molecule[i] = s.molecule[i] < 0 ? -1 - i : s.molecule[i];
    std::vector<Vec3> sites(ns);
    for (int i = 0; i < ns; i++) {
        for (int p : s.siteParticles[i]) sites[i] += pos[p];
        sites[i] = sites[i] / double(s.siteParticles[i].size());
    }
    auto delta = [&](int i, int j) { return s.periodic ? periodicDelta(sites[i], sites[j], box) : sites[j] - sites[i]; };
    double cutoff2 = s.cutoff * s.cutoff;
    // Neighbor lists (j > i).  A cell list supplies candidates for large systems; the test is the reference's.
    std::vector<std::vector<int>> nbr(ns);
    PairSettings ps;
    ps.method = s.periodic ? 2 : 1;
    ps.cutoff = s.cutoff;
    std::vector<std::pair<int, int>> cand;
    bool cellsOk = true;
    if (s.periodic) {
        // the cell search needs the cutoff below a third of the box; otherwise candidatePairs takes all pairs
        cellsOk = isRectangular(box);
    }
    if (cellsOk) candidatePairs(ns, sites, box, ps, cand);
    else
        for (int i = 0; i < ns; i++)
            for (int j = i + 1; j < ns; j++) cand.push_back({i, j});
    for (auto& c : cand) {
        int i = c.first, j = c.second;
        if (molecule[i] == molecule[j]) continue;
        Vec3 d = delta(i, j);
        if (d.dot(d) < cutoff2) nbr[i].push_back(j);
    }
    for (auto& v : nbr) std::sort(v.begin(), v.end());
    std::vector<Vec3> siteForces(ns);
    double energy = 0;
    int64_t count = 0;
    bool useDamping = (s.dampingMethod == 1);
    for (int i = 0; i < ns; i++) {
        const std::vector<int>& ni = nbr[i];
        for (size_t jj = 0; jj < ni.size(); jj++) {
            int j = ni[jj];
            const std::vector<int>& nj = nbr[j];
            for (size_t kk = jj + 1; kk < ni.size(); kk++) {
                int k = ni[kk];
                if (!std::binary_search(nj.begin(), nj.end(), k)) continue;
                double c9 = s.scale * computeC9(s.alpha[i], s.frequency[i], s.alpha[j], s.frequency[j], s.alpha[k],
                                                s.frequency[k]);
                if (s.alch[i] || s.alch[j] || s.alch[k]) c9 *= lambda;
                if (c9 == 0) continue;
                count++;
                double rates[3] = {2 * s.dampingScale / (s.width[i] + s.width[j]),
                                   2 * s.dampingScale / (s.width[i] + s.width[k]),
                                   2 * s.dampingScale / (s.width[j] + s.width[k])};
                const double et = computeTripleT<double>(delta(i, j), delta(i, k), delta(j, k), c9,
                                                         useDamping ? rates : nullptr, siteForces[i], siteForces[j],
                                                         siteForces[k], s.centroidRadius);
                energy += et;
                lastAbsEnergy() += std::fabs(et);
                if (ops) {
                    OpCounter& oc = opCounter();
                    oc = OpCounter();
                    Vec3 dummy[3];
                    computeTripleT<Counted>(delta(i, j), delta(i, k), delta(j, k), c9, useDamping ? rates : nullptr,
                                            dummy[0], dummy[1], dummy[2], s.centroidRadius);
                    // C9 (12 operations, InteraxThreeBodyForceImpl.h:69-72) and the three displacements (9)
                    ops->arith += oc.arith + 12 + 9;
                    ops->transcendental += oc.transcendental;
                }
            }
        }
    }
    for (int i = 0; i < ns; i++) {
        Vec3 f = siteForces[i] / double(s.siteParticles[i].size());
        for (int p : s.siteParticles[i]) forces[p] += f;
    }
    if (numTriples) *numTriples = count;
    return energy;
}

}  // namespace ixo

// ----------------------------------------------------------------------------------------------------------------------
// C interface for ctypes
// ----------------------------------------------------------------------------------------------------------------------
using namespace ixo;

extern "C" {

static void toVectors(int n, const double* xyz, const double* box9, std::vector<Vec3>& pos, Vec3 box[3]) {
    pos.resize(n);
    for (int i = 0; i < n; i++) pos[i] = Vec3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    for (int k = 0; k < 3; k++)
        box[k] = box9 ? Vec3(box9[3 * k], box9[3 * k + 1], box9[3 * k + 2]) : Vec3(k == 0, k == 1, k == 2);
}

static PairSettings toSettings(const ox_pair_settings* s) {
    PairSettings out;
    out.method = s->method;
    out.cutoff = s->cutoff;
    out.useSwitch = s->use_switch != 0;
    out.switchDistance = s->switch_distance;
    out.softcoreRadius = s->softcore_radius;
    for (int i = 0; i < s->num_exclusions; i++) out.exclusions.push_back({s->exclusions[2 * i], s->exclusions[2 * i + 1]});
    return out;
}

static char g_error[512];

const char* ox_last_error() { return g_error; }

// Sum of |pair energies| (before switching) or |triple energies| of the last ox_pair_force / ox_three_body call.
double ox_last_abs_energy() { return lastAbsEnergy(); }

// Energy of one pair force; forces (n x 3) are added to.  term: 0 dispersion (params n x 5: m1 m2 m3 alpha width),
// 1 exchange (n x 2: amplitude width), 2 short range (n x 3: k l width).  Returns NaN on error.
double ox_pair_force(int term, int n, const double* xyz, const double* box9, const ox_pair_settings* settings,
                     const double* params, const unsigned char* alch, double damping_scale, int use_lrc,
                     int overlap_method, double lambda, double* forces, long long* num_interacting) {
    try {
        std::vector<Vec3> pos, f(n);
        Vec3 box[3];
        toVectors(n, xyz, box9, pos, box);
        PairParams p;
        p.stride = term == 0 ? 5 : (term == 1 ? 2 : 3);
        p.p.assign(params, params + size_t(n) * p.stride);
        p.alch.assign(alch, alch + n);
        p.dampingScale = damping_scale;
        p.useLongRangeCorrection = use_lrc != 0;
        p.overlapMethod = overlap_method;
        int64_t cnt = 0;
        double e = computePairForce(PairTerm(term), pos, box, toSettings(settings), p, lambda, f, &cnt);
        if (forces)
            for (int i = 0; i < n; i++) {
                forces[3 * i] += f[i].x;
                forces[3 * i + 1] += f[i].y;
                forces[3 * i + 2] += f[i].z;
            }
        if (num_interacting) *num_interacting = cnt;
        return e;
    }
    catch (const std::exception& ex) {
        std::snprintf(g_error, sizeof(g_error), "%s", ex.what());
        return NAN;
    }
}

// Long range correction coefficients of a dispersion force.
void ox_long_range_coefficients(int n, const ox_pair_settings* settings, const double* params,
                                const unsigned char* alch, double damping_scale, int use_lrc, double* coef,
                                double* alch_coef) {
    PairParams p;
    p.stride = 5;
    p.p.assign(params, params + size_t(n) * 5);
    p.alch.assign(alch, alch + n);
    p.dampingScale = damping_scale;
    p.useLongRangeCorrection = use_lrc != 0;
    longRangeCorrection(toSettings(settings), p, *coef, *alch_coef);
}

// Energy of a three-body force; forces (n x 3) are added to.  site_params: num_sites x 3 (alpha, frequency, width).
double ox_three_body(int n, const double* xyz, const double* box9, int num_sites, const int* site_offsets,
                     const int* site_particles, const double* site_params, const int* molecule,
                     const unsigned char* alch, double cutoff, double scale, int damping_method,
                     double damping_scale, double centroid_radius, int periodic, double lambda, double* forces,
                     long long* num_triples) {
    try {
        std::vector<Vec3> pos, f(n);
        Vec3 box[3];
        toVectors(n, xyz, box9, pos, box);
        ThreeBodySettings s;
        s.siteParticles.resize(num_sites);
        for (int i = 0; i < num_sites; i++)
            s.siteParticles[i].assign(site_particles + site_offsets[i], site_particles + site_offsets[i + 1]);
        for (int i = 0; i < num_sites; i++) {
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
        int64_t cnt = 0;
        double e = computeThreeBody(pos, box, s, lambda, f, &cnt);
        if (forces)
            for (int i = 0; i < n; i++) {
                forces[3 * i] += f[i].x;
                forces[3 * i + 1] += f[i].y;
                forces[3 * i + 2] += f[i].z;
            }
        if (num_triples) *num_triples = cnt;
        return e;
    }
    catch (const std::exception& ex) {
        std::snprintf(g_error, sizeof(g_error), "%s", ex.what());
        return NAN;
    }
}

// Operations of the reference algorithm per interacting pair of one pair term (only the term's own function; the
// geometry, switch and force accumulation shared by the fused terms are ox_pair_driver_ops()).  out[0] arithmetic,
// out[1] transcendental, out[2] number of pairs.
void ox_pair_ops(int term, int n, const double* xyz, const double* box9, const ox_pair_settings* settings,
                 const double* params, const unsigned char* alch, double damping_scale, int overlap_method,
                 double lambda, double* out) {
    std::vector<Vec3> pos, f(n);
    Vec3 box[3];
    toVectors(n, xyz, box9, pos, box);
    PairParams p;
    p.stride = term == 0 ? 5 : (term == 1 ? 2 : 3);
    p.p.assign(params, params + size_t(n) * p.stride);
    p.alch.assign(alch, alch + n);
    p.dampingScale = damping_scale;
    p.overlapMethod = overlap_method;
    int64_t cnt = 0;
    OpCounter ops;
    computePairForce(PairTerm(term), pos, box, toSettings(settings), p, lambda, f, &cnt, &ops);
    out[0] = double(ops.arith);
    out[1] = double(ops.transcendental);
    out[2] = double(cnt);
}

// Per-pair operations of the pair driver (ReferenceInteraxPairIxn.h:89-126) once per pair: displacement (3),
// r^2 (5), sqrt (1 transcendental), cutoff test (1), scale and dE/dr / r (2), force vector (3), accumulation into
// both particles (6).  out[0] arithmetic, out[1] transcendental.
void ox_pair_driver_ops(double* out) {
    out[0] = 3 + 5 + 1 + 2 + 3 + 6;
    out[1] = 1;
}

// Operations per interacting triple (computeTriple, C9, displacements).  out as ox_pair_ops.
void ox_three_body_ops(int n, const double* xyz, const double* box9, int num_sites, const int* site_offsets,
                       const int* site_particles, const double* site_params, const int* molecule,
                       const unsigned char* alch, double cutoff, double scale, int damping_method,
                       double damping_scale, double centroid_radius, int periodic, double lambda, double* out) {
    std::vector<Vec3> pos, f(n);
    Vec3 box[3];
    toVectors(n, xyz, box9, pos, box);
    ThreeBodySettings s;
    s.siteParticles.resize(num_sites);
    for (int i = 0; i < num_sites; i++)
        s.siteParticles[i].assign(site_particles + site_offsets[i], site_particles + site_offsets[i + 1]);
    for (int i = 0; i < num_sites; i++) {
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
    int64_t cnt = 0;
    OpCounter ops;
    computeThreeBody(pos, box, s, lambda, f, &cnt, &ops);
    out[0] = double(ops.arith);
    out[1] = double(ops.transcendental);
    out[2] = double(cnt);
}

// Slater overlap and its derivative (for the known-answer tests).  method: 0 Exact (double precision switch),
// 2 InteraxOrder2, 1 Exact with the single precision switch.
void ox_slater_overlap(double r, double a, double b, int method, double* s, double* ds) {
    SlaterTaylorScheme scheme = method == 0 ? SlaterTaylorScheme::accurate(true)
                              : method == 1 ? SlaterTaylorScheme::accurate(false)
                                            : SlaterTaylorScheme::interaxOrder2();
    slaterOverlap(r, a, b, scheme, *s, *ds);
}

// Tang-Toennies f_6, f_8, f_10 and derivatives.
void ox_tang_toennies(double x, double* f, double* df) { tangToenniesDamping(x, f, df); }

// The derived Taylor tables, 7 x 9 each.
void ox_overlap_taylor_table(double* value, double* deriv) {
    const OverlapTaylorTable& t = overlapTaylorTable();
    std::memcpy(value, t.value, sizeof(t.value));
    std::memcpy(deriv, t.deriv, sizeof(t.deriv));
}

}  // extern "C"
