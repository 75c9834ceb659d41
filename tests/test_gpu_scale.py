"""Parity at the benchmark's own shapes, against the FP64 oracle:

* the batched configuration: all 4,096 water clusters of 2..32 waters that the bench evaluates (its seed), every
  system compared with the oracle;
* the alchemical configuration: the 96,000-atom box (32,000 waters, 9.855 nm, pair cutoff 1.0 nm, three-body cutoff
  0.8 nm on 32,000 sites) with 30 decoupled waters, windows lambda = 0, 0.37 and 1, without a soft core (each window
  interpolated from two evaluations) and with one (R = 0.1 nm: each window's alchemical pairs evaluated).

The bar is the target's: total energy within 1e-6 relative and forces within 1e-5 relative RMS of the oracle (for the
clusters, the energy relative to the sum of |pair and triple energies|, the reference's own error scale, since a
cluster's total can nearly cancel).
"""
import numpy as np
import pytest

import pyoracle
from interaxplugin import BatchContext, Context
from interaxplugin import workloads as W
from parity import ENERGY_TOL, FORCE_RMS_TOL, errors

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def test_full_cluster_batch_against_oracle():
    systems, positions = W.cluster_set(4096, seed=1)
    batch = BatchContext(systems)
    energies, forces = batch.compute(positions)
    worst_e = worst_f = 0.0
    for k, (system, pos) in enumerate(zip(systems, positions)):
        absE = []
        e_ref, f_ref = pyoracle.evaluate(system, pos, abs_energy=absE)
        e_err, f_err = errors(energies[k].sum(), forces[k], e_ref, f_ref, max(absE[0], abs(e_ref)))
        assert e_err <= ENERGY_TOL and f_err <= FORCE_RMS_TOL, (k, e_err, f_err)
        worst_e, worst_f = max(worst_e, e_err), max(worst_f, f_err)
    print(f"4096 clusters: worst energy error {worst_e:.2e}, worst force error {worst_f:.2e}")


@pytest.mark.parametrize("softcore_radius", [0.0, 0.1])
def test_alchemical_windows_96k_against_oracle(softcore_radius):
    cfg = W.CONFIGS["96k"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=1,
                                   three_body_cutoff=cfg["three_body_cutoff"], alchemical_waters=range(30),
                                   softcore_radius=softcore_radius)
    ctx = Context(system)
    ctx.setPositions(pos)
    values = [0.0, 0.37, 1.0]
    energies, forces = ctx.computeWindows("lambda_sterics", values)
    for w, lam in enumerate(values):
        e_ref, f_ref = pyoracle.evaluate(system, pos, box, {"lambda_sterics": lam})
        e_err, f_err = errors(energies[w].sum(), forces[w], e_ref, f_ref)
        print(f"R = {softcore_radius}, lambda = {lam}: energy error {e_err:.2e}, force error {f_err:.2e}")
        assert e_err <= ENERGY_TOL, (lam, e_err)
        assert f_err <= FORCE_RMS_TOL, (lam, f_err)
