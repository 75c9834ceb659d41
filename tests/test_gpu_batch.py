"""Batched evaluation of many water clusters (ix_batch_*) against the FP64 oracle, system by system, and the same
system alone and in a mix giving identical results."""
import numpy as np
import pytest

import pyoracle
from parity import errors, FORCE_RMS_TOL, ENERGY_TOL
from interaxplugin import BatchContext, Context, OpenMMException
from interaxplugin import workloads as W

pytestmark = pytest.mark.gpu


def clusters(count, seed, min_waters=2, max_waters=32):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        system, pos, _ = W.water_cluster(int(rng.integers(min_waters, max_waters + 1)), seed=seed * 1000 + k)
        out.append((system, pos))
    return out


def test_batch_matches_oracle_per_system():
    systems = clusters(24, seed=1)
    batch = BatchContext([s for s, _ in systems])
    energies, forces = batch.compute([p for _, p in systems])
    for k, (system, pos) in enumerate(systems):
        absE = []
        e_ref, f_ref = pyoracle.evaluate(system, pos, abs_energy=absE)
        e_err, f_err = errors(energies[k].sum(), forces[k], e_ref, f_ref, max(absE[0], abs(e_ref)))
        assert e_err <= ENERGY_TOL, f"system {k}: energy error {e_err:.2e}"
        assert f_err <= FORCE_RMS_TOL, f"system {k}: force error {f_err:.2e}"
    pairs, triples = batch.getCounts()
    assert pairs > 0 and triples > 0


def test_batch_long_site_lists():
    """A 300-water cluster (site lists longer than one staging of the wide triple kernel) in a mix with small ones."""
    systems = clusters(3, seed=4) + [W.water_cluster(300, seed=5)[:2]]
    batch = BatchContext([s for s, _ in systems])
    energies, forces = batch.compute([p for _, p in systems])
    system, pos = systems[-1]
    absE = []
    e_ref, f_ref = pyoracle.evaluate(system, pos, abs_energy=absE)
    e_err, f_err = errors(energies[-1].sum(), forces[-1], e_ref, f_ref, max(absE[0], abs(e_ref)))
    assert e_err <= ENERGY_TOL and f_err <= FORCE_RMS_TOL, (e_err, f_err)
    alone = BatchContext([system])
    e1, f1 = alone.compute([pos])
    assert np.array_equal(e1[0], energies[-1]) and np.array_equal(f1[0], forces[-1])


def test_batch_alone_and_in_mix_identical():
    systems = clusters(16, seed=2)
    mix = BatchContext([s for s, _ in systems])
    e_mix, f_mix = mix.compute([p for _, p in systems])
    for k in (0, 7, 15):
        alone = BatchContext([systems[k][0]])
        e1, f1 = alone.compute([systems[k][1]])
        assert np.array_equal(e1[0], e_mix[k])
        assert np.array_equal(f1[0], f_mix[k])
    # a second evaluation of new positions replays the graph
    moved = [p + 0.001 for _, p in systems]
    e2, f2 = mix.compute(moved)
    for k in (3, 9):
        alone = BatchContext([systems[k][0]])
        e1, f1 = alone.compute([moved[k]])
        assert np.array_equal(e1[0], e2[k])
        assert np.array_equal(f1[0], f2[k])


@pytest.mark.parametrize("waters,seed", [(32, 7)])
def test_batch_total_energy_bar(waters, seed):
    """The bar of the Context's cluster test: 1e-6 of the total energy, 1e-5 RMS forces, against the oracle.  (Small
    clusters whose terms cancel to a small total are judged on the reference's own scale, the sum of |energies|, in
    test_batch_matches_oracle_per_system; the Context's error on them is the same.)"""
    system, pos, _ = W.water_cluster(waters, seed=seed)
    batch = BatchContext([system])
    e, f = batch.compute([pos])
    e_ref, f_ref = pyoracle.evaluate(system, pos)
    ctx = Context(system)
    ctx.setPositions(pos)
    st = ctx.getState()
    e_ctx, _ = errors(st.getPotentialEnergy(), st.getForces(), e_ref, f_ref)
    e_err, f_err = errors(e[0].sum(), f[0], e_ref, f_ref)
    assert e_err < ENERGY_TOL and f_err < FORCE_RMS_TOL, (e_err, f_err, e_ctx)


def test_batch_rejects_mixed_settings():
    a, pa, _ = W.water_cluster(3, seed=1)
    b, pb, _ = W.water_cluster(3, seed=2)
    b.getForce(0).setSoftcoreRadius(0.1)
    batch = BatchContext([a, b])
    with pytest.raises(OpenMMException):
        batch.compute([pa, pb])
