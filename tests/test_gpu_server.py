"""Served requests (ix_server_*) and batched MD (ix_batch_md_run).

A served request's result must be the same as the request run alone: bitwise, since a periodic request runs the
context's own kernels and a batched system's evaluation does not depend on the other systems of its cohort.  The
stream mixes periodic water boxes (contexts) with water clusters (cohorts) and step counts from 0 to 8.
"""
import numpy as np
import pytest

import pyoracle
from parity import errors, ENERGY_TOL, FORCE_RMS_TOL
from interaxplugin import BatchContext, Context, Server
from interaxplugin import workloads as W

pytestmark = pytest.mark.gpu

DT = 0.0005


def _box(num_waters, seed):
    length = W.box_length_for(num_waters)
    system, pos, _ = W.water_box(num_waters, length, min(0.9, 0.45 * length), seed=seed, three_body_cutoff=0.6)
    return system, pos


def _cluster(num_waters, seed):
    system, pos, _ = W.water_cluster(num_waters, seed=seed)
    return system, pos


def _requests(seed=3, boxes=4, clusters=18):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(boxes):
        s, p = _box(int(rng.integers(230, 420)), seed=100 + k)
        out.append((s, p, W.initial_velocities(s, 300.0, seed=k), int(rng.integers(0, 9))))
    for k in range(clusters):
        s, p = _cluster(int(rng.integers(2, 33)), seed=200 + k)
        out.append((s, p, W.initial_velocities(s, 300.0, seed=50 + k), int(rng.integers(0, 9))))
    order = rng.permutation(len(out))
    return [out[i] for i in order]


def _serve(requests, **kw):
    srv = Server(**kw)
    ids = [srv.submit(s, p, v, steps=n, dt=DT) for s, p, v, n in requests]
    res = srv.run_all(timeout=120)
    stats = srv.stats()
    srv.close()
    return [res[i] for i in ids], stats


def test_batch_md_alone_and_in_mix():
    systems = [_cluster(w, seed=300 + w) for w in (3, 8, 17, 30, 5)]
    steps = [0, 4, 7, 2, 7]
    vel = [W.initial_velocities(s, 300.0, seed=k) for k, (s, _) in enumerate(systems)]
    mix = BatchContext([s for s, _ in systems])
    pos_m, vel_m, frc_m, en_m = mix.runVelocityVerlet(steps, DT, [p for _, p in systems], vel)
    for k in (0, 2, 4):
        alone = BatchContext([systems[k][0]])
        p1, v1, f1, e1 = alone.runVelocityVerlet([steps[k]], DT, [systems[k][1]], [vel[k]])
        assert np.array_equal(p1[0], pos_m[k]) and np.array_equal(v1[0], vel_m[k])
        assert np.array_equal(f1[0], frc_m[k]) and np.array_equal(e1[0], en_m[k])
    # the same trajectory as a Context's velocity Verlet: FP32 pair arithmetic in another order, so forces agree to
    # ~1e-6 relative and positions after two 0.5 fs steps to well below 1e-7 nm
    ctx = Context(systems[3][0])
    ctx.setPositions(systems[3][1])
    p2, v2, _ = ctx.runVelocityVerlet(steps[3], DT, vel[3])
    assert np.abs(p2 - pos_m[3]).max() < 1e-7
    assert np.abs(v2 - vel_m[3]).max() < 1e-4 * max(np.abs(v2).max(), 1.0)
    assert np.array_equal(pos_m[0], systems[0][1])   # zero steps: unmoved


def test_server_results_same_alone_and_in_mix():
    reqs = _requests()
    mixed, stats = _serve(reqs)
    assert all(r.status == 0 for r in mixed), [r.error for r in mixed if r.status]
    assert stats["completed"] == len(reqs) and stats["cohorts"] >= 1 and stats["contexts"] >= 1
    for k in range(len(reqs)):
        if k % 4 and k not in (1, 2):
            continue
        alone, _ = _serve([reqs[k]])
        a, m = alone[0], mixed[k]
        assert np.array_equal(a.positions, m.positions), k
        assert np.array_equal(a.velocities, m.velocities), k
        assert np.array_equal(a.forces, m.forces), k
        assert np.array_equal(a.term_energies, m.term_energies), k
    assert all(r.latency > 0 for r in mixed)


def test_server_context_requests_match_context_md():
    s, p = _box(300, seed=7)
    v = W.initial_velocities(s, 300.0, seed=1)
    (res,), _ = _serve([(s, p, v, 6)])
    ctx = Context(s)
    ctx.setPositions(p)
    pos, vel, _ = ctx.runVelocityVerlet(6, DT, v)
    assert np.array_equal(res.positions, pos) and np.array_equal(res.velocities, vel)
    st = ctx.getState()
    assert np.array_equal(res.forces, st.getForces())
    assert res.energy == pytest.approx(st.getPotentialEnergy(), rel=1e-12)


def test_server_zero_steps_against_oracle():
    reqs = [(*_cluster(12, seed=11), None, 0), (*_box(250, seed=12), None, 0)]
    results, _ = _serve(reqs)
    for (system, pos, _, _), r in zip(reqs, results):
        box = np.asarray(system.getDefaultPeriodicBoxVectors()) if system.getForce(0).getNonbondedMethod() == 2 \
            else None
        absE = []
        e_ref, f_ref = pyoracle.evaluate(system, pos, box, abs_energy=absE)
        e_err, f_err = errors(r.energy, r.forces, e_ref, f_ref, max(absE[0], abs(e_ref)))
        assert e_err <= ENERGY_TOL and f_err <= FORCE_RMS_TOL, (e_err, f_err)
        assert np.array_equal(r.positions, pos)


def test_server_admission_budget():
    """A budget that holds about two box requests: all requests finish, the reserved and arena bytes never pass the
    budget, and a request that can never fit fails with its own status."""
    reqs = [(*_box(300 + 20 * k, seed=400 + k), None, 2) for k in range(6)]
    budget = 40e6
    results, stats = _serve(reqs, budget_bytes=budget)
    assert all(r.status == 0 for r in results), [r.error for r in results if r.status]
    assert stats["peak_reserved_bytes"] <= budget and stats["peak_arena_bytes"] <= budget
    big = [(*_box(2000, seed=9), None, 0)]
    results, stats = _serve(big, budget_bytes=budget)
    assert results[0].status == 5 and "budget" in results[0].error


def test_server_reuses_contexts_of_the_same_system():
    """Requests of one System that come one after the other run on the same pooled context (its arrays, lists and
    graphs kept from the previous request), with results bitwise equal to the request run on a new server."""
    s, p = _box(300, seed=21)
    reqs = [(s, p, W.initial_velocities(s, 300.0, seed=k), 3 + k % 3) for k in range(4)]
    srv = Server()
    got = []
    for system, pos, vel, n in reqs:
        rid = srv.submit(system, pos, vel, steps=n, dt=DT)
        got.append(srv.run_all(timeout=120)[rid])
    stats = srv.stats()
    srv.close()
    assert all(r.status == 0 for r in got), [r.error for r in got]
    assert stats["contexts_reused"] >= 3, stats
    for req, m in zip(reqs, got):
        (a,), _ = _serve([req])
        assert np.array_equal(a.positions, m.positions) and np.array_equal(a.velocities, m.velocities)
        assert np.array_equal(a.forces, m.forces) and np.array_equal(a.term_energies, m.term_energies)
