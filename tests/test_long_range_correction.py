"""The long-range dispersion correction of the library (host FP64, ix_dispersion_long_range_correction) against the
FP64 oracle's restatement of the reference's quadrature (openmmapi/src/InteraxDispersionForceImpl.cpp:49-149).

The library integrates the undamped tail in closed form and the damping correction and the switching interval by
tanh-sinh quadrature; the reference uses a 32-point Gauss-Legendre rule in u = rc/r.  Both approximate the same
integrals, so they must agree far below the reference's own bar for the correction (ASSERT_EQUAL_REL 1e-9 between its
quadrature and its test integrator, tests/TestInteraxDispersionForce.h:177-225).  No GPU is needed.
"""
import numpy as np
import pytest

import pyoracle
from interaxplugin import InteraxDispersionForce
from interaxplugin import workloads as W
from interaxplugin.context import calcLongRangeCorrection

TOL = 1e-12


def _force(cutoff, switch, damping, types, alchemical=2, n=8, seed=0):
    f = InteraxDispersionForce()
    f.setNonbondedMethod(InteraxDispersionForce.CutoffPeriodic)
    f.setCutoffDistance(cutoff)
    f.setUseLongRangeCorrection(True)
    if switch is not None:
        f.setUseSwitchingFunction(True)
        f.setSwitchingDistance(switch)
    f.setDampingScale(damping)
    for i in range(n):
        f.addParticle(*types[i % len(types)], i < alchemical)
    return f


def _types(seed, count=3):
    rng = np.random.default_rng(seed)
    return [(rng.uniform(1, 3), rng.uniform(0.01, 0.1), rng.uniform(1e-3, 5e-3), rng.uniform(5e-4, 2e-3),
             rng.uniform(0.02, 0.05)) for _ in range(count)]


def _close(a, b, tol=TOL):
    for x, y in zip(a, b):
        assert abs(x - y) <= tol * max(abs(y), 1e-300), (a, b)


@pytest.mark.parametrize("cutoff,switch,damping", [(0.6, None, 1.0), (0.6, 0.45, 1.0), (0.9, None, 0.8),
                                                   (1.0, 0.75, 1.0), (0.5, None, 0.5), (1.2, 0.9, 1.3),
                                                   (0.7, 0.525, 0.3)])
def test_against_oracle(cutoff, switch, damping):
    f = _force(cutoff, switch, damping, _types(int(cutoff * 100) + int(damping * 10)))
    _close(calcLongRangeCorrection(f), pyoracle.long_range_coefficients(f))


def test_water_box_parameters():
    system, pos, box = W.water_box(216, 1.865, 0.9, seed=11, three_body=False)
    f = system.getForce(0)
    coef, alch = calcLongRangeCorrection(f)
    ref = pyoracle.long_range_coefficients(f)
    _close((coef, alch), ref)
    assert coef < 0 and alch == 0.0


def _high_precision(force):
    """The correction by 40-digit adaptive quadrature over every particle pair (mpmath), independent of both."""
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 40
    P, A = force._params_array(), force._alch_array()
    rc, beta = mp.mpf(force.getCutoffDistance()), mp.mpf(force.getDampingScale())
    sw = mp.mpf(force.getSwitchingDistance()) if force.getUseSwitchingFunction() else rc

    def energy(r, p, q):
        pref = p[3] * q[3] / max(p[3] * q[0] + q[3] * p[0], 1e-30)
        c = (pref * p[0] * q[0], 1.5 * pref * (p[0] * q[1] + p[1] * q[0]),
             pref * (2 * (p[0] * q[2] + p[2] * q[0]) + 4.2 * p[1] * q[1]))
        x = 2 * beta / (mp.mpf(p[4]) + mp.mpf(q[4])) * r
        return -sum(mp.mpf(cn) * mp.gammainc(n + 1, 0, x, regularized=True) / r ** n for n, cn in zip((6, 8, 10), c))

    sums = [mp.mpf(0), mp.mpf(0)]
    n = len(P)
    for i in range(n):
        for j in range(i, n):
            integral = mp.quad(lambda r: r * r * energy(r, P[i], P[j]), [rc, mp.inf])
            if sw < rc:
                integral += mp.quad(lambda r: r * r * energy(r, P[i], P[j]) *
                                    (lambda x: x ** 3 * (10 - 15 * x + 6 * x * x))((r - sw) / (rc - sw)), [sw, rc])
            sums[bool(A[i] or A[j])] += integral
    norm = 2 * mp.pi * n * n / (0.5 * n * (n + 1))
    return float(norm * sums[0]), float(norm * sums[1])


def test_alchemical_split_and_weak_damping():
    # x = k r of order 1 at the cutoff, where the damping matters most in the tail.  Here the reference's 32-point
    # rule is itself off by ~1e-7 (its nodes do not resolve the damping near u = 1); the library matches a 40-digit
    # integration, and the oracle within the energy bar of the parity tests.
    f = _force(0.6, 0.45, 0.05, _types(5), alchemical=3, n=6)
    coef, alch = calcLongRangeCorrection(f)
    _close((coef, alch), _high_precision(f), 1e-12)
    _close((coef, alch), pyoracle.long_range_coefficients(f), 1e-6)
    assert alch != 0.0
    # every pair with an alchemical particle goes to the alchemical part: with all particles alchemical, all of it
    g = _force(0.6, 0.45, 0.05, _types(5), alchemical=6, n=6)
    c2, a2 = calcLongRangeCorrection(g)
    assert c2 == 0.0 and abs(a2 - (coef + alch)) <= 1e-12 * abs(a2)


def test_against_high_precision_integration():
    f = _force(0.6, 0.45, 1.0, _types(9), alchemical=1, n=5)
    _close(calcLongRangeCorrection(f), _high_precision(f), 1e-12)


def test_no_correction_without_periodic_cutoff_or_when_disabled():
    f = _force(0.6, None, 1.0, _types(1))
    f.setUseLongRangeCorrection(False)
    assert calcLongRangeCorrection(f) == (0.0, 0.0)
    f.setUseLongRangeCorrection(True)
    f.setNonbondedMethod(InteraxDispersionForce.CutoffNonPeriodic)
    assert calcLongRangeCorrection(f) == (0.0, 0.0)


def test_particles_without_polarizability_have_no_correction():
    types = _types(2, 2)
    types[1] = types[1][:3] + (0.0,) + types[1][4:]
    f = _force(0.8, None, 1.0, types, alchemical=0)
    coef, _ = calcLongRangeCorrection(f)
    only = _force(0.8, None, 1.0, [types[0]], alchemical=0, n=4)
    # the pairs of the four polarizable particles alone, renormalised from N = 4 to N = 8 pairs
    c4, _ = calcLongRangeCorrection(only)
    assert abs(coef - c4 * (64 / 36) / (16 / 10)) <= 1e-12 * abs(coef)
