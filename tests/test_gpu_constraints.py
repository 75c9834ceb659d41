"""Rigid water in the device MD loop (ix_md_set_constraints): SHAKE after the drift (Newton on each cluster's
multipliers), RATTLE's velocity stage after the second half kick (a direct solve), per cluster of constrained
particles.

The reference's ns/day comes from OpenMM's integrator on systems whose waters are rigid (tests/python/benchmark.py:
88-97 with the force field's rigid water); here the constraints keep every O-H and H-H distance of the 3-site waters
to 1e-6 nm over 1,000 steps of 1 fs, no bond stretches (velocities along the bonds vanish), and the total energy
(potential plus kinetic) stays bounded.
"""
import numpy as np
import pytest

from interaxplugin import Context
from interaxplugin import workloads as W

pytestmark = pytest.mark.gpu

DT = 0.001


def _rigid_box(seed=5, num_waters=216, box_length=1.865):
    system, pos, box = W.water_box(num_waters, box_length, 0.9, seed=seed, three_body_cutoff=0.6, rigid=True)
    return system, pos


def _bond_errors(system, pos):
    err = []
    for k in range(system.getNumConstraints()):
        a, b, d = system.getConstraintParameters(k)
        err.append(abs(np.linalg.norm(pos[a] - pos[b]) - d))
    return np.array(err)


def _bond_rates(system, pos, vel):
    out = []
    for k in range(system.getNumConstraints()):
        a, b, _ = system.getConstraintParameters(k)
        r = pos[a] - pos[b]
        out.append(abs(np.dot(vel[a] - vel[b], r)) / np.dot(r, r))
    return np.array(out)


def _kinetic(system, vel):
    m = np.array([system.getParticleMass(i) for i in range(system.getNumParticles())])
    return 0.5 * float((m[:, None] * vel ** 2).sum())


def test_rigid_water_keeps_its_geometry_and_energy():
    system, pos = _rigid_box()
    assert system.getNumConstraints() == 3 * 216
    ctx = Context(system)
    ctx.setPositions(pos)
    vel = W.initial_velocities(system, 300.0, seed=1)
    energies = []
    p, v = pos, vel
    for chunk in range(10):
        p, v, e = ctx.runVelocityVerlet(100, DT, v)
        energies.append(e + _kinetic(system, v))
        assert _bond_errors(system, p).max() < 1e-6
        assert _bond_rates(system, p, v).max() < 1e-6
    energies = np.array(energies)
    kinetic = _kinetic(system, v)
    drift = np.abs(energies - energies[0]).max()
    print(f"total energy over 1000 steps: {energies[0]:.4f} .. {energies[-1]:.4f} kJ/mol, max drift {drift:.4f}, "
          f"kinetic {kinetic:.2f}")
    assert drift < 0.02 * kinetic
    # the waters moved as rigid bodies: the molecules' centres moved, their shapes did not
    assert np.abs(p - pos).max() > 1e-3


def test_constrained_md_with_async_segments_matches_one_run():
    system, pos = _rigid_box(seed=6)
    vel = W.initial_velocities(system, 300.0, seed=2)
    a = Context(system)
    a.setPositions(pos)
    pa, va, ea = a.runVelocityVerlet(30, DT, vel)
    b = Context(system)
    b.setPositions(pos)
    p1, v1, _ = b.runVelocityVerlet(10, DT, vel)
    b.setPositions(p1)
    pb, vb, eb = b.runVelocityVerlet(20, DT, v1)
    # the same steps in two calls: only the first evaluation of the second call is recomputed (same positions)
    assert np.abs(pb - pa).max() < 1e-9 and abs(eb - ea) <= 1e-9 * abs(ea)


def test_constraint_errors():
    from interaxplugin import OpenMMException
    system, pos, _ = W.water_box(27, 1.0, 0.45, seed=7, three_body=False, rigid=True)
    system.addConstraint(0, 0, 0.1)
    with pytest.raises(OpenMMException, match="Illegal particle index"):
        Context(system)


def test_general_clusters_beside_rigid_waters():
    # waters 0 and 1 joined by an O-O constraint, waters 2 and 3 by an H-H one: clusters of 6 particles and 7
    # constraints (the general solver) beside the rigid triangles of the other waters
    system, pos = _rigid_box(seed=9)
    for a, b in ((0, 3), (7, 10)):
        system.addConstraint(a, b, float(np.linalg.norm(pos[a] - pos[b])))
    ctx = Context(system)
    ctx.setPositions(pos)
    vel = W.initial_velocities(system, 300.0, seed=4)
    energies = []
    p, v = pos, vel
    for chunk in range(4):
        p, v, e = ctx.runVelocityVerlet(50, DT, v)
        energies.append(e + _kinetic(system, v))
        assert _bond_errors(system, p).max() < 1e-6
        assert _bond_rates(system, p, v).max() < 1e-6
    assert np.abs(np.array(energies) - energies[0]).max() < 0.02 * _kinetic(system, v)


def test_too_large_cluster_is_rejected():
    from interaxplugin import OpenMMException
    system, pos, _ = W.water_box(27, 1.0, 0.45, seed=7, three_body=False, rigid=True)
    # three waters joined into one cluster of 9 particles (the limit is 8)
    system.addConstraint(0, 3, 0.3)
    system.addConstraint(3, 6, 0.3)
    with pytest.raises(OpenMMException, match="cluster of 9"):
        Context(system)
