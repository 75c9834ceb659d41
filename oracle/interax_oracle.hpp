// FP64 oracle for the InteraxFF short-range path: a CPU restatement of the plugin's Reference platform.
//
// TEST INFRASTRUCTURE ONLY.  This code is the checker that the CUDA product is compared against; it is loaded by
// tests/, by the smoke check and by bench.py's CPU-baseline leg, and by nothing else.  The product never calls it.
//
// Every function names the reference file and lines whose algorithm it restates (paths inside the reference
// project).  The arithmetic is double precision, in the same order of operations as the reference where that order
// decides the rounding (pair terms, triple terms, the long range correction).
//
// The math is templated over the value type so that tests can run it with an operation-counting type, which is how
// the algorithmic work per pair and per triple is fixed (see ox_count_* in interax_oracle.cpp).
//
// Parity is pinned: tests/test_oracle_golden.py checks it against the reference's golden export values (per-term
// energies and forces of two InteraxFF systems) and its known answers; tests/test_oracle_pair_harness.py and
// tests/test_oracle_three_body.py against independent restatements of the reference's pair-test harness (in 40-digit
// arithmetic) and of its three-body all-triples loop, with every option; tests/test_long_range_correction.py against
// high-precision quadrature.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace ixo {

// ------------------------------------------------------------------------------------------------------------------
// Scalar helpers that dispatch to std:: for double and to the counting type's overloads otherwise.
// ------------------------------------------------------------------------------------------------------------------
inline double vexp(double v) { return std::exp(v); }
inline double vsqrt(double v) { return std::sqrt(v); }
inline double vabs(double v) { return std::fabs(v); }
inline double vpow(double a, double b) { return std::pow(a, b); }
inline double vval(double v) { return v; }
// single precision, for the restatement of the CPU platform (cpu_platform.cpp), which evaluates the pair terms in float
inline float vexp(float v) { return std::exp(v); }
inline float vsqrt(float v) { return std::sqrt(v); }
inline float vabs(float v) { return std::fabs(v); }
inline float vpow(float a, float b) { return std::pow(a, b); }
inline double vval(float v) { return v; }

// A double that counts the operations performed on it: +, -, *, / and negation as arithmetic, exp, sqrt and pow as
// transcendental.  Used to fix the algorithmic work per pair and per triple.
struct OpCounter {
    long long arith = 0, transcendental = 0;
};
inline OpCounter& opCounter() {
    static thread_local OpCounter c;
    return c;
}
struct Counted {
    double v;
    Counted() : v(0) {}
    Counted(double x) : v(x) {}
};
inline Counted operator+(Counted a, Counted b) { opCounter().arith++; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { opCounter().arith++; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { opCounter().arith++; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { opCounter().arith++; return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { opCounter().arith++; return Counted(-a.v); }
inline Counted vexp(Counted a) { opCounter().transcendental++; return Counted(std::exp(a.v)); }
inline Counted vsqrt(Counted a) { opCounter().transcendental++; return Counted(std::sqrt(a.v)); }
inline Counted vpow(Counted a, Counted b) { opCounter().transcendental++; return Counted(std::pow(a.v, b.v)); }
inline double vval(Counted a) { return a.v; }

// ------------------------------------------------------------------------------------------------------------------
// Taylor coefficients of the Slater overlap integral about the width l (openmmapi/include/internal/InteraxPairTerms.h
// :87-113).  They are not copied: they are derived here from the closed form by series arithmetic.  With a = l,
// b = l (1 + t) and x = r/l,
//
//   pi l^3 e^x S = F e^x / (8 x),   F e^x = 4 b^2 (1 - e^u) / D^3 + x (1 + b e^u) / D^2,   u = x t / (1 + t),
//   D = b^2 - a^2 = t (2 + t)   (in units of l)
//
// and the coefficient of t^n of the right side is the polynomial sum_k VALUE[n][k] x^k.  The derivative table follows
// from d/dr [e^-x P(x)] = e^-x (P'(x) - P(x)) / l.
// ------------------------------------------------------------------------------------------------------------------
constexpr int kMaxTaylorOrder = 6;
constexpr int kTaylorTerms = 9;

struct OverlapTaylorTable {
    double value[kMaxTaylorOrder + 1][kTaylorTerms];
    double deriv[kMaxTaylorOrder + 1][kTaylorTerms];
};

namespace detail {
// A truncated bivariate series: c[i][k] multiplies t^i x^k.
constexpr int kT = kMaxTaylorOrder + 4;   // orders of t kept
constexpr int kX = kMaxTaylorOrder + 5;   // powers of x kept
struct Series {
    double c[kT][kX] = {};
};
inline Series mul(const Series& a, const Series& b) {
    Series r;
    for (int i = 0; i < kT; i++)
        for (int k = 0; k < kX; k++) {
            if (a.c[i][k] == 0) continue;
            for (int j = 0; i + j < kT; j++)
                for (int l = 0; k + l < kX; l++)
                    r.c[i + j][k + l] += a.c[i][k] * b.c[j][l];
        }
    return r;
}
inline Series add(const Series& a, const Series& b, double sb = 1.0) {
    Series r;
    for (int i = 0; i < kT; i++)
        for (int k = 0; k < kX; k++) r.c[i][k] = a.c[i][k] + sb * b.c[i][k];
    return r;
}
inline Series constant(double v) { Series s; s.c[0][0] = v; return s; }
// (c + t)^p as a series in t, for integer p (negative allowed, c != 0)
inline Series binomialSeries(double c, int p) {
    Series s;
    double coef = std::pow(c, p);
    for (int i = 0; i < kT; i++) {
        s.c[i][0] = coef;
        coef *= double(p - i) / double(i + 1) / c;
    }
    return s;
}
}  // namespace detail

inline OverlapTaylorTable deriveOverlapTaylorTable() {
    using namespace detail;
    // u = x t / (1 + t) = x (t - t^2 + t^3 - ...)
    Series u;
    for (int i = 1; i < kT; i++) u.c[i][1] = (i % 2 == 1 ? 1.0 : -1.0);
    // e^u = sum u^m / m!
    Series expU = constant(1.0), power = constant(1.0);
    double factorial = 1.0;
    for (int m = 1; m < kT; m++) {
        power = mul(power, u);
        factorial *= m;
        expU = add(expU, power, 1.0 / factorial);
    }
    Series b = constant(1.0);
    b.c[1][0] = 1.0;                                           // b = 1 + t
    Series b2 = mul(b, b);
    Series oneMinusExpU = add(constant(1.0), expU, -1.0);
    // A = 4 b^2 (1 - e^u) (2 + t)^-3, to be divided by t^3
    Series A = mul(mul(constant(4.0), b2), mul(oneMinusExpU, binomialSeries(2.0, -3)));
    // B = x (1 + b e^u) (2 + t)^-2, to be divided by t^2
    Series xs;
    xs.c[0][1] = 1.0;
    Series B = mul(xs, mul(add(constant(1.0), mul(b, expU)), binomialSeries(2.0, -2)));
    OverlapTaylorTable table = {};
    for (int n = 0; n <= kMaxTaylorOrder; n++) {
        // coefficient of t^n of F e^x, then divide by 8 x
        for (int k = 1; k < kX; k++) {
            double v = A.c[n + 3][k] + B.c[n + 2][k];
            if (k - 1 < kTaylorTerms) table.value[n][k - 1] = v / 8.0;
        }
        for (int k = 0; k < kTaylorTerms; k++) {
            double next = (k + 1 < kTaylorTerms ? (k + 1) * table.value[n][k + 1] : 0.0);
            table.deriv[n][k] = next - table.value[n][k];
        }
    }
    return table;
}

inline const OverlapTaylorTable& overlapTaylorTable() {
    static const OverlapTaylorTable table = deriveOverlapTaylorTable();
    return table;
}

// Where the overlap uses its Taylor expansion (InteraxPairTerms.h:115-160).
struct SlaterTaylorScheme {
    int order;
    bool aboutSmallerWidth;
    double maxDelta, maxT, maxTX;
    // Exact method, with the switch of the precision (InteraxPairTerms.h:139-147)
    static SlaterTaylorScheme accurate(bool doublePrecision) {
        return {6, true, 0.0, doublePrecision ? 0.02 : 0.2, doublePrecision ? 0.3 : 1.6};
    }
    // InteraxFF order 2 scheme (InteraxPairTerms.h:151-159): 0.01 bohr in nm
    static SlaterTaylorScheme interaxOrder2() {
        return {2, false, 0.01 * 0.0529177210903, 0.0, HUGE_VAL};
    }
};

// Overlap integral S(r; a, b) and dS/dr: InteraxPairTerms.h:167-216.  For the order 2 scheme a must be the width of
// the particle with the lower index.  Both branches are evaluated, as the reference does, and one is selected.
template <class T>
inline void slaterOverlap(T r, T a, T b, const SlaterTaylorScheme& scheme, T& overlap, T& dOverlapdR) {
    const double pi = M_PI;
    // Where the Taylor expansion about l applies (the reference evaluates both branches and selects one; only the
    // selected one is evaluated here, with the same result)
    T l = scheme.aboutSmallerWidth ? (vval(a) < vval(b) ? a : b) : a;
    T invL = T(1.0) / l;
    T delta = a + b - l - l;
    T t = delta * invL;
    T x = r * invL;
    double absT = std::fabs(vval(t));
    bool nearAbsolute = std::fabs(vval(delta)) < scheme.maxDelta;
    bool nearRelative = (absT < scheme.maxT) && (absT * vval(x) < scheme.maxTX);
    if (nearAbsolute || nearRelative) {
        const OverlapTaylorTable& table = overlapTaylorTable();
        T sumValue = T(0.0), sumDeriv = T(0.0);
        for (int n = scheme.order; n >= 0; n--) {
            T value = T(0.0), deriv = T(0.0);
            for (int k = kTaylorTerms - 1; k >= 0; k--) {
                value = value * x + T(table.value[n][k]);
                deriv = deriv * x + T(table.deriv[n][k]);
            }
            sumValue = sumValue * t + value;
            sumDeriv = sumDeriv * t + deriv;
        }
        T prefactor = vexp(-x) * invL * invL * invL / T(pi);
        overlap = prefactor * sumValue;
        dOverlapdR = prefactor * invL * sumDeriv;
        return;
    }
    // closed form: S = F / (8 pi r)
    T aa = a * a, bb = b * b;
    T d = bb - aa;
    T invD2 = T(1.0) / (d * d);
    T expA = vexp(-r / a), expB = vexp(-r / b);
    T c = T(4.0) * aa * bb * invD2 / d;
    T f = c * (expA - expB) + r * invD2 * (a * expA + b * expB);
    T dfdr = c * (expB / b - expA / a) + invD2 * (a * expA + b * expB - r * (expA + expB));
    T invR = T(1.0) / r;
    overlap = f * invR / (T(8.0) * T(pi));
    dOverlapdR = (r * dfdr - f) * invR * invR / (T(8.0) * T(pi));
}

// Tang-Toennies f_6, f_8, f_10 and their derivatives: InteraxPairTerms.h:223-253.
template <class T>
inline void tangToenniesDamping(T x, T damping[3], T dDampingdX[3]) {
    const int maxTerm = 40;
    T expX = vexp(-x);
    T term = T(1.0), partialSum = T(1.0);
    T terms[11], partialSums[11];
    terms[0] = term;
    partialSums[0] = partialSum;
    for (int k = 1; k <= 10; k++) {
        term = term * x * T(1.0 / k);
        partialSum = partialSum + term;
        terms[k] = term;
        partialSums[k] = partialSum;
    }
    T tail = T(0.0);
    for (int k = 11; k <= maxTerm; k++) {
        term = term * x * T(1.0 / k);
        tail = tail + term;
    }
    for (int i = 0; i < 3; i++) {
        int n = 6 + 2 * i;
        T series = tail;
        for (int k = n + 1; k <= 10; k++) series = series + terms[k];
        damping[i] = (vval(x) < 0.5 * (n + 1)) ? expX * series : T(1.0) - expX * partialSums[n];
        dDampingdX[i] = expX * terms[n];
    }
}

// Dispersion energy of a pair and dE/dr: InteraxPairTerms.h:267-293.
template <class T>
inline void dispersionPair(T r, T m1i, T m2i, T m3i, T alphai, T widthi, T m1j, T m2j, T m3j, T alphaj, T widthj,
                           T dampingScale, T& energy, T& dEdR) {
    T denom = alphai * m1j + alphaj * m1i;
    T prefactor = alphai * alphaj / (vval(denom) > 1e-30 ? denom : T(1e-30));
    T c[3];
    c[0] = prefactor * m1i * m1j;
    c[1] = T(1.5) * prefactor * (m1i * m2j + m2i * m1j);
    c[2] = prefactor * (T(2.0) * (m1i * m3j + m3i * m1j) + T(4.2) * m2i * m2j);
    T dxdr = T(2.0) * dampingScale / (widthi + widthj);
    T damping[3], dDampingdX[3];
    tangToenniesDamping(dxdr * r, damping, dDampingdX);
    T invR = T(1.0) / r;
    T invR2 = invR * invR;
    T invRn = invR2 * invR2 * invR2;
    energy = T(0.0);
    dEdR = T(0.0);
    for (int i = 0; i < 3; i++) {
        T n = T(double(6 + 2 * i));
        energy = energy - damping[i] * c[i] * invRn;
        dEdR = dEdR - c[i] * invRn * (dDampingdX[i] * dxdr - n * damping[i] * invR);
        invRn = invRn * invR2;
    }
}

// Exchange A_i A_j S: InteraxPairTerms.h:305-312.
template <class T>
inline void exchangePair(T r, T ai, T wi, T aj, T wj, const SlaterTaylorScheme& scheme, T& energy, T& dEdR) {
    T s, ds;
    slaterOverlap(r, wi, wj, scheme, s, ds);
    T amp = ai * aj;
    energy = amp * s;
    dEdR = amp * ds;
}

// Short-range correction (K_i+K_j)/2 St + (L_i+L_j)/2 St^2: InteraxPairTerms.h:325-337.
template <class T>
inline void shortRangePair(T r, T ki, T li, T wi, T kj, T lj, T wj, const SlaterTaylorScheme& scheme, T& energy,
                           T& dEdR) {
    T s, ds;
    slaterOverlap(r, wi, wj, scheme, s, ds);
    T ws = wi + wj;
    T norm = T(8.0 * M_PI) * ws * ws * ws;
    T st = norm * s;
    T k = T(0.5) * (ki + kj);
    T l = T(0.5) * (li + lj);
    energy = (k + l * st) * st;
    dEdR = (k + T(2.0) * l * st) * norm * ds;
}

// ------------------------------------------------------------------------------------------------------------------
// Geometry
// ------------------------------------------------------------------------------------------------------------------
struct Vec3 {
    double x = 0, y = 0, z = 0;
    Vec3() = default;
    Vec3(double a, double b, double c) : x(a), y(b), z(c) {}
    Vec3 operator+(const Vec3& o) const { return {x + o.x, y + o.y, z + o.z}; }
    Vec3 operator-(const Vec3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    Vec3 operator*(double s) const { return {x * s, y * s, z * s}; }
    Vec3 operator/(double s) const { return {x / s, y / s, z / s}; }
    Vec3& operator+=(const Vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    Vec3& operator-=(const Vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    double dot(const Vec3& o) const { return x * o.x + y * o.y + z * o.z; }
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

// Displacement to - from with the reduced-box minimum image, c then b then a: the convention of OpenMM's
// ReferenceForce::getDeltaRPeriodic used at platforms/reference/src/ReferenceInteraxPairIxn.h:94 and of
// ReferenceInteraxThreeBodyIxn.cpp:74-82.
inline Vec3 periodicDelta(const Vec3& from, const Vec3& to, const Vec3* box) {
    Vec3 d = to - from;
    d -= box[2] * std::floor(d.z / box[2].z + 0.5);
    d -= box[1] * std::floor(d.y / box[1].y + 0.5);
    d -= box[0] * std::floor(d.x / box[0].x + 0.5);
    return d;
}

// ------------------------------------------------------------------------------------------------------------------
// Pair driver: ReferenceInteraxPairIxn.h:82-128 and the kernels' pair callbacks, ReferenceInteraxKernels.cpp:79-183.
// ------------------------------------------------------------------------------------------------------------------
enum PairTerm { kDispersion = 0, kExchange = 1, kShortRange = 2 };

struct PairSettings {
    int method = 0;               // 0 NoCutoff, 1 CutoffNonPeriodic, 2 CutoffPeriodic
    double cutoff = 1.0;
    bool useSwitch = false;
    double switchDistance = -1.0;
    double softcoreRadius = 0.0;
    std::vector<std::pair<int, int>> exclusions;
};

// Candidate pairs i < j that are not excluded.  With a cutoff and a rectangular box that holds at least three cells
// per axis, a cell list is used; otherwise all pairs.  Either way the caller applies the exact r < cutoff test, so the
// interacting set is the same as the reference's voxel-hash list (ReferenceInteraxPairIxn.h:86-99).
void candidatePairs(int n, const std::vector<Vec3>& pos, const Vec3* box, const PairSettings& s,
                    std::vector<std::pair<int, int>>& out);

struct PairParams {
    // dispersion: m1, m2, m3, alpha, width; exchange: amplitude, width; short range: k, l, width
    std::vector<double> p;   // numParticles x stride
    int stride = 0;
    std::vector<uint8_t> alch;
    double dampingScale = 1.0;
    bool useLongRangeCorrection = false;
    int overlapMethod = 0;   // 0 Exact, 2 InteraxOrder2
};

double computePairForce(PairTerm term, const std::vector<Vec3>& pos, const Vec3* box, const PairSettings& s,
                        const PairParams& params, double lambda, std::vector<Vec3>& forces,
                        int64_t* numInteracting = nullptr, OpCounter* ops = nullptr);

// Long range correction coefficients: openmmapi/src/InteraxDispersionForceImpl.cpp:49-149.
void longRangeCorrection(const PairSettings& s, const PairParams& params, double& coefficient,
                         double& alchemicalCoefficient);

// ------------------------------------------------------------------------------------------------------------------
// Three-body (ATM): InteraxThreeBodyTerms.h:51-146, ReferenceInteraxThreeBodyIxn.cpp:39-135.
// ------------------------------------------------------------------------------------------------------------------
struct ThreeBodySettings {
    std::vector<std::vector<int>> siteParticles;
    std::vector<double> alpha, frequency, width;
    std::vector<int> molecule;
    std::vector<uint8_t> alch;
    double cutoff = 1.2, scale = 1.0, dampingScale = 1.0, centroidRadius = 0.0;
    int dampingMethod = 0;   // 0 NoDamping, 1 TangToennies
    bool periodic = false;
};

double computeThreeBody(const std::vector<Vec3>& pos, const Vec3* box, const ThreeBodySettings& s, double lambda,
                        std::vector<Vec3>& forces, int64_t* numTriples = nullptr, OpCounter* ops = nullptr);

// One triple in double precision (InteraxThreeBodyTerms.h:97-146): energy returned, forces added to fA, fB, fC.
double atmTriple(const Vec3& ab, const Vec3& ac, const Vec3& bc, double c9, const double* rates, Vec3& fA, Vec3& fB,
                 Vec3& fC, double centroidRadius);
double atmC9(double a1, double w1, double a2, double w2, double a3, double w3);

}  // namespace ixo

// Settings of a pair force as the C interface takes them (ctypes).
extern "C" struct ox_pair_settings {
    int method;
    double cutoff;
    int use_switch;
    double switch_distance;
    double softcore_radius;
    int num_exclusions;
    const int* exclusions;   // 2 x num_exclusions
};
