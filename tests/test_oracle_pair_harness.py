"""Pin the FP64 oracle's pair forces to the reference's pair-test harness, with every option of a pair force (no GPU).

The harness (tests/TestInteraxPairForce.h:59-148 with the three forces' test models) is restated in 40-digit
arithmetic in pair_harness.py; the cases hold exclusions, a lone pair, equal, nearly equal and distinct widths,
alchemical particles in and out of the soft core, and a periodic cutoff with switching in a rectangular and a
triclinic box, and no cutoff.
"""
import math

import numpy as np
import pytest

import pyoracle
from interaxplugin import InteraxShortRangeForce, System
from pair_harness import CASES, KINDS, MODELS, build, case_box, harness, harness_positions, mpmath, short_range_pair


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("method, lam, triclinic", CASES)
def test_pair_force_against_the_harness(kind, method, lam, triclinic):
    rng = np.random.default_rng(5)
    pos = harness_positions(rng)
    system, force = build(kind, method, rng)
    box = case_box(triclinic)
    e, f = pyoracle.evaluate(system, pos, box, parameters={force.getAlchemicalParameterName(): lam})
    expected, forces, scale = harness(force, MODELS[kind], pos, box, lam)
    # both in double or better: the oracle agrees to ~1e-13 of the error scale, where the soft core alone moves the
    # energy by a few per cent and a change of lambda by 1e-4 moves it by 1e-5
    assert abs(e - expected) <= 1e-11 * scale, (e, expected, scale)
    rms = math.sqrt((forces ** 2).mean())
    assert np.abs(f - forces).max() <= 1e-10 * rms, np.abs(f - forces).max() / rms


def short_range_system(particles):
    """A System of one InteraxShortRangeForce over the given (K, L, width) particles."""
    system = System()
    force = InteraxShortRangeForce()
    for k, l, width in particles:
        system.addParticle(1.0)
        force.addParticle(k, l, width)
    system.addForce(force)
    return system, force


def test_short_range_normalization():
    """tests/TestInteraxShortRangeForce.h:87-100: for equal widths at r -> 0 the normalized overlap St -> 1, and the
    energy is (K_i + K_j)/2 St + (L_i + L_j)/2 St^2 with St = exp(-x) (1 + x + x^2/3), x = r/s."""
    pos = np.array([[0.0, 0.0, 0.0], [1e-6, 0.0, 0.0]])
    system, _ = short_range_system([(-1000.0, 40000.0, 0.02), (-2000.0, 60000.0, 0.02)])
    e, f = pyoracle.evaluate(system, pos, np.eye(3) * 10.0)
    x = 1e-6 / 0.02
    st = math.exp(-x) * (1 + x + x * x / 3)
    assert e == pytest.approx(-1500.0 * st + 50000.0 * st * st, rel=1e-12)
    assert np.all(np.isfinite(f))


def test_short_range_zero_width():
    """tests/TestInteraxShortRangeForce.h:105-121: a particle of zero width (a lone pair) interacts with nothing."""
    pos = np.array([[0.0, 0.0, 0.0], [0.03, 0.0, 0.0], [0.0, 0.12, 0.0]])
    particles = [(-1000.0, 40000.0, 0.02), (-2000.0, 60000.0, 0.0), (500.0, 20000.0, 0.025)]
    system, _ = short_range_system(particles)
    e, f = pyoracle.evaluate(system, pos, np.eye(3) * 10.0)
    with mpmath.workdps(40):
        expected = short_range_pair(particles[0], particles[2])(mpmath.mpf("0.12"))
    assert e == pytest.approx(float(expected), rel=1e-12)
    assert np.all(f[1] == 0.0)
