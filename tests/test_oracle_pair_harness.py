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
from pair_harness import CASES, KINDS, MODELS, build, case_box, harness, harness_positions


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
