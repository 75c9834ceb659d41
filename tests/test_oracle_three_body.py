"""Pin the FP64 oracle's Axilrod-Teller-Muto term to the reference's own three-body tests (no GPU).

* testTriple (tests/TestInteraxThreeBodyForce.h:185-222): one triple against its energy written out with the law of
  cosines, three identical sites against C9 = 3/4 alpha C6, and the scale factor.
* The all-triples loop of the reference's three-body tests (tests/TestInteraxThreeBodyForce.h:71-129, restated in
  triples_loop.py) on a periodic case of every option, with the forces as central differences of its energy.
"""
import math

import numpy as np
import pytest

import pyoracle
from triples_loop import (BOX_LENGTH, CUTOFF, DAMPING_CASES, LAMBDA, SCALE, SITE_TYPES, brute_force_energy, c9_of,
                          loop_case, loop_energy_and_forces, single_sites)

TRIPLE = np.array([[0.1, -0.2, 0.05], [0.45, 0.1, -0.1], [-0.05, 0.3, 0.2]])


def test_triple_against_the_law_of_cosines():
    system, force = single_sites(SITE_TYPES)
    p = TRIPLE
    rab, rac, rbc = (np.linalg.norm(p[1] - p[0]), np.linalg.norm(p[2] - p[0]), np.linalg.norm(p[2] - p[1]))
    cos_a = (rab ** 2 + rac ** 2 - rbc ** 2) / (2 * rab * rac)
    cos_b = (rab ** 2 + rbc ** 2 - rac ** 2) / (2 * rab * rbc)
    cos_c = (rac ** 2 + rbc ** 2 - rab ** 2) / (2 * rac * rbc)
    geometry = (1 + 3 * cos_a * cos_b * cos_c) / (rab * rac * rbc) ** 3
    expected = c9_of(*[t[:2] for t in SITE_TYPES]) * geometry
    e, _ = pyoracle.evaluate(system, p, np.eye(3) * 10.0)
    assert e == pytest.approx(expected, rel=1e-12)
    # three identical sites: the C6 of a site is 3/4 alpha^2 w, and C9 = 3/4 alpha C6
    a, w, _ = SITE_TYPES[0]
    system, force = single_sites([SITE_TYPES[0]] * 3)
    c6 = 0.75 * a * a * w
    e, _ = pyoracle.evaluate(system, p, np.eye(3) * 10.0)
    assert e == pytest.approx(0.75 * a * c6 * geometry, rel=1e-12)
    # the scale factor multiplies every triple
    force.setScaleFactor(0.7)
    e_scaled, _ = pyoracle.evaluate(system, p, np.eye(3) * 10.0)
    assert e_scaled == pytest.approx(0.7 * e, rel=1e-12)


@pytest.mark.parametrize("tt_scale, radius", DAMPING_CASES)
def test_against_the_all_triples_loop(tt_scale, radius):
    system, force, sites, pos = loop_case(tt_scale, radius, np.random.default_rng(7))
    box = np.eye(3) * BOX_LENGTH
    e, f = pyoracle.evaluate(system, pos, box, parameters={force.getAlchemicalParameterName(): LAMBDA})
    expected, fd = loop_energy_and_forces(sites, pos, tt_scale, radius)
    # the case exercises the alchemical factor (some triples hold an alchemical site) and the damping
    assert expected != 0.0
    assert brute_force_energy(sites, pos, BOX_LENGTH, CUTOFF, SCALE, tt_scale, radius, 1.0) != expected
    if tt_scale or radius:
        undamped = brute_force_energy(sites, pos, BOX_LENGTH, CUTOFF, SCALE, 0.0, 0.0, LAMBDA)
        assert abs(expected - undamped) > 1e-2 * abs(undamped)
    assert e == pytest.approx(expected, rel=1e-10)
    rms = math.sqrt((fd ** 2).mean())
    assert np.abs(f - fd).max() <= 1e-6 * rms
