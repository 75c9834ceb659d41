"""The B200 kernels against the reference's test harnesses themselves, the restatements the oracle is pinned to.

The pair-test harness (tests/TestInteraxPairForce.h:59-148, in 40-digit arithmetic in pair_harness.py) with the
three pair forces in one System, so that they run in one fused pass: exclusions, a lone pair, equal, nearly equal and
distinct widths, alchemical particles in and out of the soft core, switching, rectangular and triclinic periodic
boxes, and no cutoff.  The three-body test's all-triples loop (triples_loop.py) with every option.

Each force group is held to the reference's single-precision bar for its pair tests (energy 2e-5 of the sum of |pair
energies|, force 2e-4 of the largest force, tests/TestInteraxPairForce.h:727-730); the fused total to this build's
target (1e-6 of the sum of |pair energies|, 1e-5 relative RMS force) against the FP64 oracle.
"""
import numpy as np
import pytest

import pair_harness as H
import triples_loop as T
from interaxplugin import Context, System
from parity import compare, gpu_state, max_force_error

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method, lam, triclinic", H.CASES)
def test_fused_pair_forces_against_the_harness(method, lam, triclinic):
    rng = np.random.default_rng(11)
    pos = H.harness_positions(rng)
    system = System()
    for _ in range(len(pos)):
        system.addParticle(1.0)
    forces = []
    for group, kind in enumerate(H.KINDS):
        _, force = H.build(kind, method, rng)
        force.setForceGroup(group)
        system.addForce(force)
        forces.append(force)
    box = H.case_box(triclinic)
    params = {"lambda_sterics": lam}
    ctx = Context(system)
    for group, (kind, force) in enumerate(zip(H.KINDS, forces)):
        e, f, _ = gpu_state(system, pos, box, params, groups=1 << group, context=ctx)
        expected, f_ref, scale = H.harness(force, H.MODELS[kind], pos, box, lam)
        assert abs(e - expected) <= 2e-5 * scale, (kind, e, expected, scale)
        assert max_force_error(f, f_ref) <= 2e-4, kind
    compare(system, pos, box, params, scale="abs", context=ctx)


@pytest.mark.parametrize("tt_scale, radius", T.DAMPING_CASES)
def test_three_body_against_the_all_triples_loop(tt_scale, radius):
    """The ATM kernels against the reference test's all-triples loop (tests/TestInteraxThreeBodyForce.h:71-129, restated
    in triples_loop.py): centroid sites, molecules, the cutoff, periodic images, Tang-Toennies and centroid
    damping, alchemical sites; held to the reference's three-body bar (energy 1e-5 relative, force 1e-4 of the largest,
    tests/TestInteraxThreeBodyForce.h:615-620) and to this build's target against the oracle."""
    system, force, sites, pos = T.loop_case(tt_scale, radius, np.random.default_rng(7))
    box = np.eye(3) * T.BOX_LENGTH
    params = {force.getAlchemicalParameterName(): T.LAMBDA}
    e, f, ctx = gpu_state(system, pos, box, params)
    expected, fd = T.loop_energy_and_forces(sites, pos, tt_scale, radius)
    assert abs(e - expected) <= 1e-5 * abs(expected), (e, expected)
    assert max_force_error(f, fd) <= 1e-4
    compare(system, pos, box, params, scale="abs", context=ctx)
