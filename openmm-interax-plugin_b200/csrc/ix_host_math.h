// Host-side double precision pieces of the path: the dispersion pair energy used by the long range correction and
// the correction itself.  The reference computes the correction on the host in double precision for every platform
// (openmmapi/src/InteraxDispersionForceImpl.cpp:86-149, used by CommonInteraxKernels.cpp:297 and applied at :252-258).
#pragma once

#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>
#include <vector>

namespace ixhost {

// f_n(x) = 1 - exp(-x) sum_{k<=n} x^k/k!, n = 6, 8, 10, with the series form below (n+1)/2 (InteraxPairTerms.h:223-253).
inline void tangToennies(double x, double f[3]) {
    double e = std::exp(-x);
    double terms[11], partial[11];
    double term = 1.0, sum = 1.0;
    terms[0] = partial[0] = 1.0;
    for (int k = 1; k <= 10; k++) {
        term *= x / k;
        sum += term;
        terms[k] = term;
        partial[k] = sum;
    }
    double tail = 0.0;
    for (int k = 11; k <= 40; k++) {
        term *= x / k;
        tail += term;
    }
    for (int i = 0; i < 3; i++) {
        int n = 6 + 2 * i;
        double series = tail;
        for (int k = n + 1; k <= 10; k++) series += terms[k];
        f[i] = x < 0.5 * (n + 1) ? e * series : 1.0 - e * partial[n];
    }
}

// Dispersion energy of a pair at distance r (InteraxPairTerms.h:267-293); p = m1, m2, m3, alpha, width.
inline double dispersionEnergy(double r, const double* pi, const double* pj, double beta) {
    double denom = std::max(pi[3] * pj[0] + pj[3] * pi[0], 1e-30);
    double pref = pi[3] * pj[3] / denom;
    double c6 = pref * pi[0] * pj[0];
    double c8 = 1.5 * pref * (pi[0] * pj[1] + pi[1] * pj[0]);
    double c10 = pref * (2.0 * (pi[0] * pj[2] + pi[2] * pj[0]) + 4.2 * pi[1] * pj[1]);
    double f[3];
    tangToennies(2.0 * beta / (pi[4] + pj[4]) * r, f);
    double r2 = r * r, r6 = r2 * r2 * r2;
    return -(f[0] * c6 / r6 + f[1] * c8 / (r6 * r2) + f[2] * c10 / (r6 * r2 * r2));
}

// 32-point Gauss-Legendre rule on (0, 1), nodes by Newton iteration on P_n.
inline void gaussLegendre(int n, std::vector<double>& nodes, std::vector<double>& weights) {
    nodes.resize(n);
    weights.resize(n);
    for (int i = 0; i < n; i++) {
        double x = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = x;
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

// Long range correction coefficients: E_lrc = (coefficient + lambda alchemicalCoefficient)/V.  Particles are grouped
// into classes of identical parameters; each pair of classes integrates r^2 E(r) beyond the cutoff (u = rc/r) and
// r^2 (1 - S(r)) E(r) over the switching interval; 2 pi N^2 times the average over the N(N+1)/2 pairs.
inline void longRangeCorrection(int n, const double* params, const unsigned char* alch, double cutoff, bool useSwitch,
                                double switchDistance, double beta, double& coefficient, double& alchCoefficient) {
    typedef std::tuple<double, double, double, double, double, bool> Class;
    std::map<Class, int> counts;
    for (int i = 0; i < n; i++) {
        const double* p = params + 5 * i;
        counts[std::make_tuple(p[0], p[1], p[2], p[3], p[4], alch[i] != 0)]++;
    }
    std::vector<std::pair<Class, int>> classes(counts.begin(), counts.end());
    std::vector<double> nodes, weights;
    gaussLegendre(32, nodes, weights);
    double sw = useSwitch ? switchDistance : cutoff;
    double width = cutoff - sw;
    double sum = 0.0, alchSum = 0.0;
    for (size_t i = 0; i < classes.size(); i++)
        for (size_t j = i; j < classes.size(); j++) {
            const Class& a = classes[i].first;
            const Class& b = classes[j].first;
            if (std::get<3>(a) * std::get<3>(b) == 0) continue;
            double pa[5] = {std::get<0>(a), std::get<1>(a), std::get<2>(a), std::get<3>(a), std::get<4>(a)};
            double pb[5] = {std::get<0>(b), std::get<1>(b), std::get<2>(b), std::get<3>(b), std::get<4>(b)};
            double integral = 0.0;
            for (int k = 0; k < 32; k++) {
                double u = nodes[k];
                integral += weights[k] * dispersionEnergy(cutoff / u, pa, pb, beta) * cutoff * cutoff * cutoff /
                            (u * u * u * u);
                if (useSwitch) {
                    double x = nodes[k];
                    double r = sw + x * width;
                    double oneMinusS = x * x * x * (10 + x * (-15 + x * 6));
                    integral += weights[k] * width * oneMinusS * dispersionEnergy(r, pa, pb, beta) * r * r;
                }
            }
            double na = classes[i].second, nb = classes[j].second;
            double count = (i == j ? 0.5 * na * (na + 1) : na * nb);
            if (std::get<5>(a) || std::get<5>(b)) alchSum += count * integral;
            else sum += count * integral;
        }
    double N = n;
    double norm = 2 * M_PI * N * N / (0.5 * N * (N + 1));
    coefficient = norm * sum;
    alchCoefficient = norm * alchSum;
}

}  // namespace ixhost
