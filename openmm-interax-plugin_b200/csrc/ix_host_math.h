// Host-side FP64 pieces of the dispersion force: the XDM combination of C6/C8/C10 and the long-range correction.
//
// The correction is the energy of the dispersion tail beyond the cutoff (and of the part the switching function
// removes inside it) for a uniform fluid of the System's particle classes.  Its value is defined by the reference
// (openmmapi/src/InteraxDispersionForceImpl.cpp:86-149: per pair of particle classes the integral of r^2 E(r) from
// the cutoff to infinity plus that of r^2 (1 - S(r)) E(r) over the switching interval, weighted by the number of
// class pairs and normalised as 2 pi N^2 / (N (N + 1) / 2) times their sum; E_lrc = (coef + lambda alchCoef) / V).
// The evaluation here is independent of the reference's Gauss-Legendre quadrature:
//   * the undamped tail -sum_n C_n / r^n integrates in closed form, -C_n / ((n - 3) rc^(n-3));
//   * the damping correction sum_n C_n q_n(kr) / r^n, q_n = 1 - f_n the Tang-Toennies complement, and the switching
//     interval are integrated by tanh-sinh quadrature refined until two levels agree to 1e-15;
//   * the particles are grouped into classes by sorting their parameter rows.
#pragma once

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

namespace ixhost {

// Dispersion coefficients of a pair from the particles' XDM parameters p = (m1, m2, m3, alpha, ...):
// c[0] = C6, c[1] = C8, c[2] = C10 (the combination rule of InteraxPairTerms.h:274-278, with its 1e-30 floor).
inline void xdmCoefficients(const double* p, const double* q, double c[3]) {
    const double pref = p[3] * q[3] / std::max(p[3] * q[0] + q[3] * p[0], 1e-30);
    c[0] = pref * p[0] * q[0];
    c[1] = 1.5 * pref * (p[0] * q[1] + p[1] * q[0]);
    c[2] = pref * (2.0 * (p[0] * q[2] + p[2] * q[0]) + 4.2 * p[1] * q[1]);
}

// The Tang-Toennies damping of order n, f_n(x) = P(n + 1, x) (the regularized lower incomplete gamma function), and
// its complement q_n(x) = e^-x sum_{k<=n} x^k / k!.  Below x = n + 1 the series e^-x sum_{k>n} x^k / k! gives f_n
// without cancellation (its terms fall at once); above, the finite sum gives q_n without cancellation.
inline void tangToenniesPair(int n, double x, double& f, double& q) {
    if (x <= 0.0) {
        f = 0.0;
        q = 1.0;
        return;
    }
    if (!(x < INFINITY)) {      // zero widths: no damping
        f = 1.0;
        q = 0.0;
        return;
    }
    const double e = std::exp(-x);
    if (x < n + 1.0) {
        double term = 1.0;
        for (int k = 1; k <= n; k++) term *= x / k;     // x^n / n!
        double sum = 0.0;
        for (int k = n + 1; k < n + 200; k++) {
            term *= x / k;
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        f = e * sum;
        q = 1.0 - f;
    }
    else {
        double term = 1.0, sum = 1.0;
        for (int k = 1; k <= n; k++) {
            term *= x / k;
            sum += term;
        }
        q = e * sum;
        f = 1.0 - q;
    }
}

// Integral of g over (lo, hi) by tanh-sinh quadrature (H. Takahasi and M. Mori, "Double exponential formulas for
// numerical integration", Publ. RIMS Kyoto Univ. 9, 721-741 (1974)): x = tanh(pi/2 sinh t) turns the interval into
// the real line with weights that fall doubly exponentially, so the trapezoidal rule in t converges geometrically for
// integrands analytic inside the interval, whatever they do at its ends.  The step is halved (reusing the previous
// nodes) until two levels agree to `rel`.  Nodes are placed from the nearer end of the interval, so that those
// crowding an end keep their distance to it.
template <class G>
double tanhSinh(G g, double lo, double hi, double rel = 1e-15) {
    const double half = 0.5 * (hi - lo);
    if (!(half > 0.0)) return 0.0;
    const double tMax = 4.0;       // weight beyond ~1e-36 of the centre's
    auto node = [&](double t) {
        const double s = 0.5 * M_PI * std::sinh(t);
        const double c = std::cosh(s);
        const double w = 0.5 * M_PI * std::cosh(t) / (c * c);
        // distance of the node to the interval's end, 1 - |tanh s| = 1 / (e^|s| cosh s), without cancellation
        const double edge = half / (std::exp(std::fabs(s)) * c);
        const double x = s >= 0.0 ? hi - edge : lo + edge;
        return half * w * g(x);
    };
    double h = 0.5;
    double sum = node(0.0);
    for (double t = h; t <= tMax; t += h) sum += node(t) + node(-t);
    double value = h * sum;
    for (int level = 0; level < 12; level++) {
        h *= 0.5;
        for (double t = h; t <= tMax; t += 2.0 * h) sum += node(t) + node(-t);
        const double next = h * sum;
        const bool done = std::fabs(next - value) <= rel * std::fabs(next);
        value = next;
        if (done && level >= 1) break;
    }
    return value;
}

// Damped dispersion energy of a pair at r with coefficients c and damping rate k (x = k r).
inline double dampedDispersion(double r, const double c[3], double k) {
    double e = 0.0, rn = r * r * r * r * r * r;
    for (int i = 0; i < 3; i++) {
        double f, q;
        tangToenniesPair(6 + 2 * i, k * r, f, q);
        e -= c[i] * f / rn;
        rn *= r * r;
    }
    return e;
}

// Integral of r^2 E(r) from the cutoff to infinity plus that of r^2 (1 - S(r)) E(r) over the switching interval, for
// one pair of classes (coefficients c, damping rate k).
inline double tailIntegral(const double c[3], double k, double cutoff, bool useSwitch, double switchDistance) {
    // undamped tail, closed form
    double total = 0.0, rcPow = cutoff * cutoff * cutoff;
    for (int i = 0; i < 3; i++) {
        total -= c[i] / ((3.0 + 2.0 * i) * rcPow);
        rcPow *= cutoff * cutoff;
    }
    // damping correction beyond the cutoff, in u = rc / r on (0, 1): r^2 dr = rc^3 u^-4 du
    if (k > 0.0 && k < INFINITY) {
        total += tanhSinh(
            [&](double u) {
                if (u < 1e-6) return 0.0;    // q_n(k rc / u) < e^-(k rc 1e6): nothing left
                const double r = cutoff / u;
                double sum = 0.0, rn = r * r * r * r * r * r;
                for (int i = 0; i < 3; i++) {
                    double f, q;
                    tangToenniesPair(6 + 2 * i, k * r, f, q);
                    sum += c[i] * q / rn;
                    rn *= r * r;
                }
                return sum * r * r * cutoff / (u * u);
            },
            0.0, 1.0);
    }
    // the part of the interaction the switching function removes inside the cutoff
    if (useSwitch && switchDistance < cutoff) {
        const double width = cutoff - switchDistance;
        total += tanhSinh(
            [&](double r) {
                const double x = (r - switchDistance) / width;
                const double removed = x * x * x * (10.0 + x * (-15.0 + 6.0 * x));   // 1 - S
                return r * r * removed * dampedDispersion(r, c, k);
            },
            switchDistance, cutoff);
    }
    return total;
}

// Long-range correction coefficients of a dispersion force: E_lrc = (coefficient + lambda alchCoefficient) / V.
// params: n x 5 (m1, m2, m3, alpha, width) per particle; alch: n flags.  beta: the damping scale.
inline void longRangeCorrection(int n, const double* params, const unsigned char* alch, double cutoff,
                                bool useSwitch, double switchDistance, double beta, double& coefficient,
                                double& alchCoefficient) {
    coefficient = alchCoefficient = 0.0;
    if (n <= 0) return;
    // classes: particles whose parameter rows and alchemical flags are equal, found by sorting the rows
    auto less = [&](int a, int b) {
        for (int d = 0; d < 5; d++)
            if (params[5 * (size_t)a + d] != params[5 * (size_t)b + d])
                return params[5 * (size_t)a + d] < params[5 * (size_t)b + d];
        return (alch[a] != 0) < (alch[b] != 0);
    };
    auto same = [&](int a, int b) {
        for (int d = 0; d < 5; d++)
            if (params[5 * (size_t)a + d] != params[5 * (size_t)b + d]) return false;
        return (alch[a] != 0) == (alch[b] != 0);
    };
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), less);
    std::vector<int> rep;             // a particle of each class
    std::vector<double> count;        // its size
    for (int k = 0; k < n; k++) {
        if (k == 0 || !same(order[k - 1], order[k])) {
            rep.push_back(order[k]);
            count.push_back(0.0);
        }
        count.back() += 1.0;
    }
    double plain = 0.0, alchemical = 0.0;
    const size_t numClasses = rep.size();
    for (size_t a = 0; a < numClasses; a++)
        for (size_t b = a; b < numClasses; b++) {
            const double* p = params + 5 * (size_t)rep[a];
            const double* q = params + 5 * (size_t)rep[b];
            if (p[3] * q[3] == 0.0) continue;       // a class without polarizability has no dispersion
            double c[3];
            xdmCoefficients(p, q, c);
            const double ws = p[4] + q[4];
            const double k = ws != 0.0 ? 2.0 * beta / ws : INFINITY;   // x = k r; zero widths leave f_n = 1
            // class pairs: unordered pairs of distinct particles plus the self pairs, na (na + 1) / 2 within a class
            const double pairs = a == b ? 0.5 * count[a] * (count[a] + 1.0) : count[a] * count[b];
            const double value = pairs * tailIntegral(c, k, cutoff, useSwitch, switchDistance);
            if (alch[rep[a]] || alch[rep[b]]) alchemical += value;
            else plain += value;
        }
    const double N = n;
    const double norm = 2.0 * M_PI * N * N / (0.5 * N * (N + 1.0));
    coefficient = norm * plain;
    alchCoefficient = norm * alchemical;
}

}  // namespace ixhost
