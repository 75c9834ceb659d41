"""Alchemical windows: one context evaluated at many values of lambda_sterics (ix_compute_windows).

Each window must match the context evaluated at that value with setParameter + getState and the FP64 oracle at the
same value (InteraxPairForce.cpp:138-146 define the parameter; the pair kernels scale pairs with one alchemical
particle, kernels/interaxPairForce.cu, and the three-body kernel scales triples with an alchemical site,
kernels/interaxThreeBodyForce.cu).  Without a soft core the energies and forces are linear in lambda and the windows
come from two evaluations; with a soft core the pair terms are evaluated once at 0 and each window adds its alchemical
pairs (the same pair kernel and terms), within the same tolerances of getState at that value.
"""
import numpy as np
import pytest

import pyoracle
from interaxplugin import Context
from interaxplugin import workloads as W
from parity import ENERGY_TOL, FORCE_RMS_TOL, errors

pytestmark = pytest.mark.gpu

WINDOWS = np.linspace(0.0, 1.0, 16)


def _system(softcore_radius, seed=3, three_body=True):
    cfg = W.CONFIGS["small"]
    return W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=seed,
                       three_body_cutoff=cfg["three_body_cutoff"], alchemical_waters=range(12),
                       softcore_radius=softcore_radius, three_body=three_body)


def _per_window(ctx, values):
    out_e, out_f = [], []
    for lam in values:
        ctx.setParameter("lambda_sterics", lam)
        st = ctx.getState()
        out_e.append(st.getTermEnergies().copy())
        out_f.append(st.getForces().copy())
    return np.array(out_e), np.array(out_f)


@pytest.mark.parametrize("softcore_radius", [0.0, 0.15])
@pytest.mark.parametrize("three_body", [True, False])
def test_windows_match_get_state(softcore_radius, three_body):
    system, pos, box = _system(softcore_radius, three_body=three_body)
    ctx = Context(system)
    ctx.setPositions(pos)
    ctx.setParameter("lambda_sterics", 0.8)
    for repeat in range(2):          # the second pass replays the cached window graphs
        energies, forces = ctx.computeWindows("lambda_sterics", WINDOWS)
        assert energies.shape == (len(WINDOWS), 4) and forces.shape == (len(WINDOWS), len(pos), 3)
        assert ctx.getParameter("lambda_sterics") == 0.8
    ref_e, ref_f = _per_window(ctx, WINDOWS)
    for w in range(len(WINDOWS)):
        e_err, f_err = errors(energies[w].sum(), forces[w], ref_e[w].sum(), ref_f[w],
                              abs_energy=np.abs(ref_e[w]).sum())
        assert e_err <= ENERGY_TOL and f_err <= FORCE_RMS_TOL, (w, e_err, f_err)
        assert np.allclose(energies[w], ref_e[w], rtol=1e-6, atol=1e-6 * np.abs(ref_e[w]).sum())


@pytest.mark.parametrize("softcore_radius", [0.0, 0.15])
def test_windows_against_oracle(softcore_radius):
    system, pos, box = _system(softcore_radius, seed=1)
    ctx = Context(system)
    ctx.setPositions(pos)
    values = [0.0, 0.37, 1.0]
    energies, forces = ctx.computeWindows("lambda_sterics", values)
    for w, lam in enumerate(values):
        e_ref, f_ref = pyoracle.evaluate(system, pos, box, {"lambda_sterics": lam})
        e_err, f_err = errors(energies[w].sum(), forces[w], e_ref, f_ref)
        assert e_err <= ENERGY_TOL, (lam, e_err)
        assert f_err <= FORCE_RMS_TOL, (lam, f_err)


def test_windows_restore_state_and_energy_only():
    system, pos, box = _system(0.0)
    ctx = Context(system)
    ctx.setPositions(pos)
    before = ctx.getState()
    energies = ctx.computeWindows("lambda_sterics", [0.25, 0.5], getForces=False)
    assert energies.shape == (2, 4)
    after = ctx.getState()
    assert after.getPotentialEnergy() == before.getPotentialEnergy()
    assert np.array_equal(after.getForces(), before.getForces())
    # a parameter no force uses: every window is the plain evaluation
    plain = ctx.computeWindows("lambda_unused", [0.0, 0.5, 1.0], getForces=False)
    for w in range(3):
        assert abs(plain[w].sum() - before.getPotentialEnergy()) <= 1e-12 * abs(before.getPotentialEnergy())
    assert "lambda_unused" not in ctx.getParameters()
    assert ctx.computeWindows("lambda_sterics", []).__len__() == 2
