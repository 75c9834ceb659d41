"""Neighbor-list overflow and growth on every path, forced by small list capacities (ix_set_list_capacity).

OpenMM recomputes forces whose neighbor list overflowed after growing it, and the reference's three-body kernel scans
every later site for a site whose list overflowed (platforms/common/src/kernels/interaxThreeBody.cc:111-112,
437-438).  No call here may return forces that miss interactions: each forced run is compared with the same run at
the default capacity (bitwise where the same kernels run) and with the FP64 oracle.
"""
import ctypes

import numpy as np
import pytest

import pyoracle
from interaxplugin import Context, Server, _capi
from interaxplugin import workloads as W
from parity import ENERGY_TOL, FORCE_RMS_TOL, errors

pytestmark = pytest.mark.gpu

DT = 0.001


def _small(seed=4):
    cfg = W.CONFIGS["small"]
    return W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=seed,
                       three_body_cutoff=cfg["three_body_cutoff"])


def _state(system, pos, capacity=None):
    ctx = Context(system)
    if capacity:
        ctx.setListCapacity(*capacity)
    ctx.setPositions(pos)
    st = ctx.getState()
    return ctx, st.getTermEnergies().copy(), st.getForces().copy()


def test_pair_list_overflow_grows_and_recomputes():
    system, pos, box = _small()
    _, e_ref, f_ref = _state(system, pos)
    ctx, e, f = _state(system, pos, (8, 0))
    tiles, _, _ = ctx.getListStats()
    assert tiles > 8
    assert np.array_equal(f, f_ref)
    assert np.allclose(e, e_ref, rtol=1e-13, atol=0)
    # this box's terms cancel 18-fold in the total, so the energy is compared on the reference's own error scale
    # (the sum of |pair and triple energies|); the forced overflow's result is bitwise the unforced one above
    absE = []
    e_or, f_or = pyoracle.evaluate(system, pos, box, abs_energy=absE)
    e_err, f_err = errors(e.sum(), f, e_or, f_or, max(absE[0], abs(e_or)))
    assert e_err <= ENERGY_TOL and f_err <= FORCE_RMS_TOL


def test_three_body_list_overflow_scans_the_sites():
    system, pos, box = _small()
    atm_group = 1 << system.getForce(3).getForceGroup()
    ref = Context(system)
    ref.setPositions(pos)
    st = ref.getState(groups=atm_group)
    ctx = Context(system)
    ctx.setListCapacity(0, 2)
    ctx.setPositions(pos)
    first = ctx.getState(groups=atm_group)          # sites with more than 2 later neighbors scan every later site
    _, sites, _ = ctx.getListStats()
    assert sites > 2
    second = ctx.getState(groups=atm_group)         # the grown lists
    for s in (first, second):
        e_err, f_err = errors(s.getPotentialEnergy(), s.getForces(), st.getPotentialEnergy(), st.getForces())
        assert e_err <= 1e-6 and f_err <= 1e-5, (e_err, f_err)
    assert ctx.getCounts()[1] == ref.getCounts()[1]
    e_or, f_or = pyoracle.evaluate(system, pos, box, groups=atm_group)
    e_err, f_err = errors(first.getPotentialEnergy(), first.getForces(), e_or, f_or)
    assert e_err <= ENERGY_TOL and f_err <= FORCE_RMS_TOL


def test_md_pair_overflow_reruns_the_steps():
    system, pos, _ = _small(seed=6)
    vel = W.initial_velocities(system, 300.0, seed=1)
    a = Context(system)
    a.setPositions(pos)
    pa, va, ea = a.runVelocityVerlet(12, DT, vel)
    b = Context(system)
    b.setListCapacity(8, 0)
    b.setPositions(pos)
    pb, vb, eb = b.runVelocityVerlet(12, DT, vel)
    assert b.getListStats()[2] >= 1                 # the steps were rerun after the list grew
    assert np.array_equal(pb, pa) and np.array_equal(vb, va) and eb == ea


def test_md_async_segments_rerun_after_overflow():
    system, pos, _ = _small(seed=7)
    vel = W.initial_velocities(system, 300.0, seed=2)
    masses = _capi.arr([system.getParticleMass(i) for i in range(system.getNumParticles())], np.float64)
    L = _capi.lib()
    out = []
    for capacity in (None, (8, 0)):
        ctx = Context(system)
        if capacity:
            ctx.setListCapacity(*capacity)
        ctx.setPositions(pos)
        ctx._check(L.ix_md_set_masses(ctx._ctx, _capi.ptr(masses)))
        p = pos.copy()
        v = _capi.arr(vel, np.float64).copy()
        e = ctypes.c_double()
        ctx._check(L.ix_md_run(ctx._ctx, 0, DT, _capi.ptr(p), _capi.ptr(v), ctypes.byref(e)))
        # two segments with different time steps, then one finish
        ctx._check(L.ix_md_steps_async(ctx._ctx, 5, DT))
        ctx._check(L.ix_md_steps_async(ctx._ctx, 4, 0.5 * DT))
        ctx._check(L.ix_md_finish(ctx._ctx, _capi.ptr(p), _capi.ptr(v), ctypes.byref(e)))
        out.append((p, v, e.value, ctx.getListStats()[2]))
    assert out[1][3] >= 1
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1]) and out[0][2] == out[1][2]


def test_md_three_body_overflow_needs_no_rerun():
    system, pos, _ = _small(seed=8)
    vel = W.initial_velocities(system, 300.0, seed=3)
    a = Context(system)
    a.setPositions(pos)
    pa, va, ea = a.runVelocityVerlet(6, DT, vel)
    b = Context(system)
    b.setListCapacity(0, 2)
    b.setPositions(pos)
    pb, vb, eb = b.runVelocityVerlet(6, DT, vel)
    assert b.getListStats()[2] == 0
    assert np.abs(pb - pa).max() < 1e-9
    assert abs(eb - ea) <= 1e-6 * abs(ea)


def test_served_request_overflow():
    system, pos, _ = _small(seed=9)
    vel = W.initial_velocities(system, 300.0, seed=4)
    srv = Server(budget_bytes=2e9)
    ids = [srv.submit(system, pos, vel, steps=5, dt=DT, list_capacity=cap) for cap in (None, (8, 0), (0, 2))]
    res = srv.run_all(timeout=120)
    srv.close()
    plain, pair, site = (res[i] for i in ids)
    for r in (plain, pair, site):
        assert r.status == 0, r.error
    # a pair-list overflow reruns the request from its description: the same trajectory
    assert np.array_equal(pair.positions, plain.positions) and np.array_equal(pair.forces, plain.forces)
    # a three-body list overflow keeps the run: the same trajectory up to the rounding of the scanned sites
    assert np.abs(site.positions - plain.positions).max() < 1e-9
    e_err, f_err = errors(site.energy, site.forces, plain.energy, plain.forces)
    assert e_err <= 1e-6 and f_err <= 1e-5
