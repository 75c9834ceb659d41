"""Parity of the B200 kernels with the FP64 oracle and with the reference's golden export values.

Every test calls the CUDA path through the C ABI (interaxplugin.Context -> libinterax_b200.so) and checks it against
the oracle on the same inputs.  The cases follow the reference's own tests (tests/TestInteraxPairForce.h:701-714,
TestInteraxDispersionForce.h, TestInteraxExchangeForce.h, TestInteraxShortRangeForce.h,
TestInteraxThreeBodyForce.h:604-637, TestInteraxExportValues.h:188-197).

Tolerances: the target of this build is 1e-6 relative total energy and 1e-5 relative RMS force against the FP64
oracle.  Single pairs and triples are checked against the reference's single-precision tolerances for those tests
(energy 2e-5 of sum |E_pair|, force 2e-4 of the largest force; three-body 1e-5 / 1e-4), since a lone pair's energy
may be a near-cancellation of terms.
"""
import ctypes
import math

import numpy as np
import pytest

import pyoracle
from golden_systems import load_golden, TERM_NAMES
from interaxplugin import (Context, System, InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                           InteraxThreeBodyForce, OpenMMException)
from interaxplugin import workloads as W
from parity import compare, errors, gpu_state, max_force_error

pytestmark = pytest.mark.gpu

PAIR_E_TOL, PAIR_F_TOL = 2e-5, 2e-4        # tests/TestInteraxPairForce.h:727-730 (single precision)
ATM_E_TOL, ATM_F_TOL = 1e-5, 1e-4          # tests/TestInteraxThreeBodyForce.h:615-620


# ------------------------------------------------------------------------------------------------------------------
# golden export values (tests/TestInteraxExportValues.h)
# ------------------------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["cluster", "methanol_box"])
@pytest.mark.parametrize("exact", [True, False])
def test_export_values(name, exact):
    system, positions, box, expected = load_golden(name)
    if exact:
        for f in system._forces:
            if hasattr(f, "setOverlapMethod"):
                f.setOverlapMethod(0)
    ctx = Context(system)
    ctx.setPeriodicBoxVectors(*box)
    ctx.setPositions(positions)
    for group, term in enumerate(TERM_NAMES):
        st = ctx.getState(groups=1 << group)
        e, f = st.getPotentialEnergy(), st.getForces()
        E, F = expected[term]
        rms = math.sqrt((F ** 2).sum() / F.size)
        # the reference's single-precision bar for the export (Exact: 2e-6 energy, 5e-5 x RMS force); the order-2
        # scheme is held to the same bar here because the kernel's overlap does not lose precision outside it
        assert abs(e - E) <= 2e-6 * abs(E), (term, e, E)
        assert np.abs(f - F).max() <= 5e-5 * rms, term
        # and against the oracle at this build's target
        e_ref, f_ref = pyoracle.evaluate(system, positions, box, groups=1 << group)
        e_err, f_err = errors(e, f, e_ref, f_ref)
        assert e_err <= 1e-6 and f_err <= 1e-5, (term, e_err, f_err)


# ------------------------------------------------------------------------------------------------------------------
# pair-force models of the reference tests
# ------------------------------------------------------------------------------------------------------------------
DISP_TYPES = [
    (2.0412491330659432, 0.07991696226413432, 0.003917538949072952, 0.0020393931939312773, 0.026844933830306183),
    (2.179116829570064, 0.05077216863583387, 0.001421435052885423, 0.0012613225562556841, 0.021090413137365274),
    (0.47385034770767653, 0.0062664158577877644, 0.00015411387998271836, 0.00023498508736915282, 0.020351567997950105),
    (3.9405044694974447, 0.18787610923101286, 0.010735264902054127, 0.004221894603968141, 0.03096091246647922)]
EXCH_TYPES = [(10.326424719450545, 0.0248302193400194), (1.0254403205662432, 0.019763296864870033),
              (13.231601566169132, 0.02761867008817038), (1.5623921585722147, 0.021706271973167678)]
SR_TYPES = [(-1102.281886852146, 5953.779066676866, 0.017966632940037853),
            (1236.5568512540217, 80470.88690318535, 0.026044362132579005),
            (-1579.591012686484, 70439.46596886561, 0.027056173026181088),
            (-1702.373363056105, 47202.476121472, 0.01880253891316055)]


def make_force(kind):
    if kind == "dispersion":
        f = InteraxDispersionForce()
        f.setDampingScale(0.7155241370201111)
    elif kind == "exchange":
        f = InteraxExchangeForce()
    else:
        f = InteraxShortRangeForce()
    return f


def add_typed(f, kind, t, alch=False):
    if kind == "dispersion":
        f.addParticle(*DISP_TYPES[t], isAlchemical=alch)
    elif kind == "exchange":
        f.addParticle(*EXCH_TYPES[t], isAlchemical=alch)
    else:
        f.addParticle(*SR_TYPES[t], isAlchemical=alch)


def typed_system(kind, types, alch=None):
    system = System()
    f = make_force(kind)
    for k, t in enumerate(types):
        system.addParticle(1.0)
        add_typed(f, kind, t, bool(alch[k]) if alch else False)
    system.addForce(f)
    return system, f


KINDS = ["dispersion", "exchange", "short_range"]


@pytest.mark.parametrize("kind", KINDS)
def test_pair_energies(kind):
    """tests/TestInteraxPairForce.h:169-193: every pair of types over a range of distances."""
    direction = np.array([0.3, -0.5, 0.8]) / math.sqrt(0.98)
    for t1 in range(4):
        for t2 in range(t1, 4):
            system, f = typed_system(kind, [t1, t2])
            ctx = Context(system)
            for r in (0.06, 0.1, 0.15, 0.2, 0.25, 0.3, 0.4, 0.5, 0.7):
                pos = np.array([[0.1, 0.2, -0.1], [0.1, 0.2, -0.1]]) + np.array([[0, 0, 0], direction * r])
                e_ref, f_ref = pyoracle.evaluate(system, pos)
                e, frc, _ = gpu_state(system, pos, context=ctx)
                assert abs(e - e_ref) <= PAIR_E_TOL * abs(e_ref), (t1, t2, r, e, e_ref)
                assert max_force_error(frc, f_ref) <= PAIR_F_TOL, (t1, t2, r)


@pytest.mark.parametrize("kind", KINDS)
def test_exclusions(kind):
    system, f = typed_system(kind, [0, 1, 2, 3, 0])
    f.addExclusion(0, 1)
    f.addExclusion(3, 2)
    f.addExclusion(4, 0)
    pos = np.array([[0, 0, 0], [0.25, 0, 0], [0, 0.3, 0], [0.1, 0.1, 0.2], [-0.2, 0.05, 0.1]])
    compare(system, pos, energy_tol=PAIR_E_TOL, force_tol=PAIR_F_TOL, scale="abs")


@pytest.mark.parametrize("kind", KINDS)
def test_cutoff(kind):
    system, f = typed_system(kind, [0, 1, 2])
    f.setNonbondedMethod(InteraxDispersionForce.CutoffNonPeriodic)
    f.setCutoffDistance(0.35)
    compare(system, np.array([[0, 0, 0], [0.2, 0, 0], [0.45, 0, 0]]), energy_tol=PAIR_E_TOL, force_tol=PAIR_F_TOL,
            scale="abs")
    e, frc, _ = gpu_state(system, np.array([[0, 0, 0], [0.36, 0, 0], [0, 0.36, 0.36]]))
    assert e == 0.0 and np.all(frc == 0.0)


@pytest.mark.parametrize("kind", KINDS)
def test_periodic(kind):
    system, f = typed_system(kind, [0, 1, 3])
    f.setNonbondedMethod(InteraxDispersionForce.CutoffPeriodic)
    f.setCutoffDistance(0.5)
    box = np.diag([1.2, 1.1, 1.3])
    system.setDefaultPeriodicBoxVectors(*box)
    pos = np.array([[0.05, 0.5, 0.6], [1.1, 0.55, 0.6], [0.1, 1.05, 2.6 + 0.05]])
    compare(system, pos, box, energy_tol=PAIR_E_TOL, force_tol=PAIR_F_TOL, scale="abs")


@pytest.mark.parametrize("kind", KINDS)
def test_triclinic(kind):
    """tests/TestInteraxPairForce.h:280-311: 50 particles spread over several periodic copies of a triclinic box."""
    box = np.array([[2.0, 0, 0], [0.4, 2.1, 0], [-0.5, 0.7, 1.9]])
    rng = np.random.default_rng(5)
    system, f = typed_system(kind, [i % 4 for i in range(50)])
    f.setNonbondedMethod(InteraxDispersionForce.CutoffPeriodic)
    f.setCutoffDistance(0.75)
    system.setDefaultPeriodicBoxVectors(*box)
    pos = []
    while len(pos) < 50:
        p = box[0] * (3 * rng.random() - 1) + box[1] * (3 * rng.random() - 1) + box[2] * (3 * rng.random() - 1)
        ok = True
        for q in pos:
            d = p - q
            d -= box[2] * round(d[2] / box[2][2])
            d -= box[1] * round(d[1] / box[1][1])
            d -= box[0] * round(d[0] / box[0][0])
            if d @ d < 0.12 ** 2:
                ok = False
        if ok:
            pos.append(p)
    compare(system, np.array(pos), box, energy_tol=PAIR_E_TOL, force_tol=PAIR_F_TOL, scale="abs")


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("method", [1, 2])
def test_switching_function(kind, method):
    system, f = typed_system(kind, [0, 2])
    f.setNonbondedMethod(method)
    f.setCutoffDistance(0.5)
    f.setUseSwitchingFunction(True)
    f.setSwitchingDistance(0.3)
    box = np.diag([2.0, 2.0, 2.0])
    system.setDefaultPeriodicBoxVectors(*box)
    ctx = Context(system)
    for r in np.arange(0.25, 0.55, 0.02):
        pos = np.array([[0, 0, 0], [0, r, 0]])
        e_ref, f_ref = pyoracle.evaluate(system, pos, box)
        e, frc, _ = gpu_state(system, pos, box, context=ctx)
        # near the cutoff S(r) is small: errors relative to the unswitched pair (tests/TestInteraxPairForce.h:330-336)
        g = make_force(kind)
        add_typed(g, kind, 0)
        add_typed(g, kind, 2)
        e0 = pyoracle.pair_force(pyoracle.term_of(g), g, pos, box)[0] if r < 0.5 else 0.0
        assert abs(e - e_ref) <= PAIR_E_TOL * abs(e0) + 1e-12, r
        assert np.abs(frc - f_ref).max() <= PAIR_F_TOL * (abs(e0) / 0.2 + np.abs(f_ref).max()) + 1e-12, r


@pytest.mark.parametrize("kind", KINDS)
def test_alchemical(kind):
    system, f = typed_system(kind, [0, 1, 2, 3, 1], alch=[1, 1, 0, 0, 0])
    f.setAlchemicalParameterName("lambda_test")
    pos = np.array([[0, 0, 0], [0.2, 0, 0], [0, 0.25, 0], [0.15, 0.2, 0.15], [-0.1, 0.1, 0.25]])
    ctx = Context(system)
    assert ctx.getParameter("lambda_test") == 1.0
    for lam in (1.0, 0.0, 0.3, 0.8):
        e_ref, f_ref = pyoracle.evaluate(system, pos, parameters={"lambda_test": lam})
        e, frc, _ = gpu_state(system, pos, parameters={"lambda_test": lam}, context=ctx)
        assert abs(e - e_ref) <= PAIR_E_TOL * max(abs(e_ref), 1.0), lam
        assert max_force_error(frc, f_ref) <= PAIR_F_TOL, lam


@pytest.mark.parametrize("kind", KINDS)
def test_softcore(kind):
    system, f = typed_system(kind, [0, 1, 2, 3], alch=[1, 1, 0, 0])
    f.setSoftcoreRadius(0.2)
    f.setNonbondedMethod(InteraxDispersionForce.CutoffNonPeriodic)
    f.setCutoffDistance(0.6)
    f.setUseSwitchingFunction(True)
    f.setSwitchingDistance(0.4)
    pos = np.array([[0, 0, 0], [0.18, 0, 0], [0.02, 0.1, 0], [0.3, 0.25, 0.15]])
    ctx = Context(system)
    for lam in (1.0, 0.7, 0.2, 0.0):
        e_ref, f_ref = pyoracle.evaluate(system, pos, parameters={"lambda_sterics": lam})
        e, frc, _ = gpu_state(system, pos, parameters={"lambda_sterics": lam}, context=ctx)
        assert abs(e - e_ref) <= PAIR_E_TOL * max(abs(e_ref), 1.0), lam
        assert max_force_error(frc, f_ref) <= PAIR_F_TOL, lam


def _molecule_positions(num_molecules, box_size, seed, offsets, min_sep):
    rng = np.random.default_rng(seed)
    box = np.diag([box_size] * 3)
    pos = []
    while len(pos) < num_molecules * len(offsets):
        origin = rng.random(3) * box_size
        mol = [origin + np.array(o) for o in offsets]
        ok = True
        for p in pos:
            for q in mol:
                d = p - q
                d -= box_size * np.round(d / box_size)
                ok &= d @ d > min_sep ** 2
        if ok:
            pos += mol
    return np.array(pos), box


@pytest.mark.parametrize("kind", KINDS)
def test_large_system(kind):
    """tests/TestInteraxPairForce.h:421-471: 60 triatomic molecules, every option of the force."""
    pos, box = _molecule_positions(60, 2.3, 0, [(0, 0, 0), (0.1, 0, 0), (0, 0.1, 0)], 0.2)
    types = [(i + j) % 4 for i in range(60) for j in range(3)]
    alch = [1 if i < 4 else 0 for i in range(60) for j in range(3)]
    system, f = typed_system(kind, types, alch)
    system.setDefaultPeriodicBoxVectors(*box)
    f.setNonbondedMethod(InteraxDispersionForce.CutoffPeriodic)
    f.setCutoffDistance(0.9)
    f.setUseSwitchingFunction(True)
    f.setSwitchingDistance(0.75)
    f.setSoftcoreRadius(0.15)
    for i in range(60):
        for j in range(3):
            for k in range(j):
                f.addExclusion(3 * i + k, 3 * i + j)
    ctx = Context(system)
    for lam in (1.0, 0.4):
        compare(system, pos, box, {"lambda_sterics": lam}, context=ctx, scale="abs")


@pytest.mark.parametrize("kind", KINDS)
def test_changing_parameters(kind):
    system, f = typed_system(kind, [0, 1, 2, 3], alch=[0, 0, 1, 0])
    pos = np.array([[0, 0, 0], [0.2, 0, 0], [0, 0.22, 0], [0.15, 0.2, 0.15]])
    ctx = Context(system)
    e1, _, _ = gpu_state(system, pos, parameters={"lambda_sterics": 0.5}, context=ctx)
    if kind == "dispersion":
        f.setParticleParameters(1, 2.5, 0.06, 0.002, 0.0015, 0.023, False)
        f.setDampingScale(0.8)
    elif kind == "exchange":
        f.setParticleParameters(1, 2.0, 0.023, False)
        f.setParticleParameters(3, 5.0, 0.026, False)
    else:
        f.setParticleParameters(1, 900.0, 50000.0, 0.024, False)
        f.setParticleParameters(3, -1000.0, 30000.0, 0.02, False)
    f.updateParametersInContext(ctx)
    e2, _, _, _, _ = compare(system, pos, parameters={"lambda_sterics": 0.5}, context=ctx, energy_tol=PAIR_E_TOL,
                             force_tol=PAIR_F_TOL, scale="abs")
    assert abs(e1 - e2) > 1e-3 * abs(e1)


@pytest.mark.parametrize("kind", KINDS)
def test_illegal_settings(kind):
    system, f = typed_system(kind, [0, 1])
    system.addParticle(1.0)
    with pytest.raises(OpenMMException, match="exactly as many particles"):
        Context(system)
    system, f = typed_system(kind, [0, 1])
    f.addExclusion(0, 2)
    with pytest.raises(OpenMMException, match="Illegal particle index for an exclusion"):
        Context(system)
    system, f = typed_system(kind, [0, 1])
    f.setNonbondedMethod(1)
    f.setCutoffDistance(0.5)
    f.setUseSwitchingFunction(True)
    f.setSwitchingDistance(0.5)
    with pytest.raises(OpenMMException, match="Switching distance"):
        Context(system)
    system, f = typed_system(kind, [0, 1])
    f.setNonbondedMethod(2)
    f.setCutoffDistance(1.1)
    system.setDefaultPeriodicBoxVectors((2, 0, 0), (0, 3, 0), (0, 0, 3))
    with pytest.raises(OpenMMException, match="half the periodic box"):
        Context(system)


def test_exchange_equal_widths_and_zero_width():
    """tests/TestInteraxExchangeForce.h:110-154."""
    system = System()
    for _ in range(2):
        system.addParticle(1.0)
    f = InteraxExchangeForce()
    f.addParticle(2.0, 0.025)
    f.addParticle(3.0, 0.025)
    system.addForce(f)
    ctx = Context(system)
    for r in (0.02, 0.1, 0.3):
        x = r / 0.025
        e, frc, _ = gpu_state(system, np.array([[0, 0, 0], [r, 0, 0]]), context=ctx)
        expected = 6.0 * math.exp(-x) * (1 + x + x * x / 3) / (64 * math.pi * 0.025 ** 3)
        dedr = -6.0 * math.exp(-x) * x * (1 + x) / 3 / (64 * math.pi * 0.025 ** 4)
        assert e == pytest.approx(expected, rel=PAIR_E_TOL)
        assert frc[1][0] == pytest.approx(-dedr, rel=PAIR_F_TOL)
    system = System()
    for _ in range(3):
        system.addParticle(1.0)
    f = InteraxExchangeForce()
    f.addParticle(2.0, 0.025)
    f.addParticle(3.0, 0.0)
    f.addParticle(1.5, 0.02)
    system.addForce(f)
    e, frc, _ = gpu_state(system, np.array([[0, 0, 0], [0.03, 0, 0], [0, 0.2, 0]]))
    assert e == pytest.approx(3.0 * pyoracle.slater_overlap(0.2, 0.025, 0.02)[0], rel=PAIR_E_TOL)
    assert np.all(frc[1] == 0.0)


def test_overlap_methods():
    """tests/TestInteraxPairForce.h:580-630, compared with the FP64 oracle: the Exact method in float is held to
    3e-5 as the reference, and the order-2 scheme is tested in float too (the reference skips it)."""
    width = 0.02
    for method in (0, 2):
        for diff in (0.0, 2e-4, 1e-3, 0.005, 0.01, 0.05, 0.12, 0.3, 0.5):
            for order in (0, 1):
                widths = [width, width * (1 + diff)]
                system = System()
                for _ in range(2):
                    system.addParticle(1.0)
                f = InteraxExchangeForce()
                f.addParticle(3.0, widths[order])
                f.addParticle(3.0, widths[1 - order])
                f.setOverlapMethod(method)
                system.addForce(f)
                ctx = Context(system)
                for r in (0.03, 0.06, 0.1, 0.15, 0.2, 0.3):
                    pos = np.array([[0, 0, 0], [0, 0, r]])
                    e_ref, f_ref = pyoracle.evaluate(system, pos)
                    e, frc, _ = gpu_state(system, pos, context=ctx)
                    assert abs(e - e_ref) <= 3e-5 * abs(e_ref), (method, diff, order, r)
                    assert abs(frc[1][2] - f_ref[1][2]) <= 3e-4 * abs(f_ref[1][2]), (method, diff, order, r)


@pytest.mark.parametrize("method", [0, 2])
def test_overlap_methods_against_reference(method):
    """tests/TestInteraxPairForce.h:638-695: 150 molecules of four particles with nearly equal widths."""
    widths = [0.02, 0.02 * (1 + 0.004), 0.02 * (1 + 0.1), 0.026]
    pos, box = _molecule_positions(150, 2.0, 1, [(0, 0, 0), (0.1, 0, 0), (0, 0.1, 0), (0, 0, 0.1)], 0.12)
    for kind in ("exchange", "short_range"):
        system = System()
        system.setDefaultPeriodicBoxVectors(*box)
        f = make_force(kind)
        for i in range(150):
            system.addParticle(1.0)
            system.addParticle(1.0)
            system.addParticle(1.0)
            system.addParticle(1.0)
            for j in range(4):
                if kind == "exchange":
                    f.addParticle(3.0, widths[j])
                else:
                    f.addParticle(-1500.0, 60000.0, widths[j])
            for j in range(4):
                for k in range(j + 1, 4):
                    f.addExclusion(4 * i + j, 4 * i + k)
        f.setNonbondedMethod(2)
        f.setCutoffDistance(0.6)
        f.setOverlapMethod(method)
        system.addForce(f)
        compare(system, pos, box, scale="abs")


def test_combined_pair_forces():
    """tests/TestInteraxShortRangeForce.h:127-210: the three forces together, in one group and in separate groups."""
    rng = np.random.default_rng(2)
    box_size = 1.8
    box = np.diag([box_size] * 3)
    pos = []
    while len(pos) < 80:
        origin = rng.random(3) * box_size
        mol = [origin, origin + np.array([0.1, 0, 0])]
        ok = True
        for p in pos:
            for q in mol:
                d = p - q
                d -= box_size * np.round(d / box_size)
                ok &= d @ d > 0.2 ** 2
        if ok:
            pos += mol
    pos = np.array(pos)

    def create(same_group):
        system = System()
        system.setDefaultPeriodicBoxVectors(*box)
        d, x, s = InteraxDispersionForce(), InteraxExchangeForce(), InteraxShortRangeForce()
        for i in range(40):
            alch = i == 0
            system.addParticle(1.0)
            system.addParticle(1.0)
            d.addParticle(*DISP_TYPES[0], isAlchemical=alch)
            d.addParticle(*DISP_TYPES[2], isAlchemical=alch)
            x.addParticle(*EXCH_TYPES[0], isAlchemical=alch)
            x.addParticle(*EXCH_TYPES[1], isAlchemical=alch)
            s.addParticle(*SR_TYPES[0], isAlchemical=alch)
            s.addParticle(*SR_TYPES[3], isAlchemical=alch)
        for k, f in enumerate((d, x, s)):
            for i in range(40):
                f.addExclusion(2 * i, 2 * i + 1)
            f.setNonbondedMethod(2)
            f.setCutoffDistance(0.8)
            f.setUseSwitchingFunction(True)
            f.setSwitchingDistance(0.7)
            f.setSoftcoreRadius(0.1)
            f.setForceGroup(0 if same_group else k)
            system.addForce(f)
        d.setUseLongRangeCorrection(True)
        return system

    sep, comb = create(False), create(True)
    params = {"lambda_sterics": 0.6}
    e1, f1, _, _, ctx1 = compare(sep, pos, box, params, scale="abs")
    e2, f2, _, _, _ = compare(comb, pos, box, params, scale="abs")
    assert abs(e1 - e2) <= 1e-6 * abs(e1)
    for k in range(3):
        compare(sep, pos, box, params, groups=1 << k, context=ctx1, scale="abs")


# ------------------------------------------------------------------------------------------------------------------
# three-body (tests/TestInteraxThreeBodyForce.h)
# ------------------------------------------------------------------------------------------------------------------
SITE_TYPES = [(0.004087456746801944, 911.0681141195369, 0.03), (0.0016246535729804365, 1262.664320774599, 0.025),
              (0.008817709933796472, 747.5256543931184, 0.035)]


def single_sites(n):
    system = System()
    f = InteraxThreeBodyForce()
    for i in range(n):
        system.addParticle(1.0)
        a, w, s = SITE_TYPES[i % 3]
        f.addSite([i], a, w, s)
    system.addForce(f)
    return system, f


def test_atm_triple():
    system, f = single_sites(3)
    pos = np.array([[0.1, -0.2, 0.05], [0.45, 0.1, -0.1], [-0.05, 0.3, 0.2]])
    compare(system, pos, energy_tol=ATM_E_TOL, force_tol=1e-5, scale="abs")
    rab, rac, rbc = (np.linalg.norm(pos[1] - pos[0]), np.linalg.norm(pos[2] - pos[0]), np.linalg.norm(pos[2] - pos[1]))
    ca = (rab ** 2 + rac ** 2 - rbc ** 2) / (2 * rab * rac)
    cb = (rab ** 2 + rbc ** 2 - rac ** 2) / (2 * rab * rbc)
    cc = (rac ** 2 + rbc ** 2 - rab ** 2) / (2 * rac * rbc)
    (aA, wA, _), (aB, wB, _), (aC, wC, _) = SITE_TYPES
    c9 = 1.5 * aA * aB * aC * wA * wB * wC * (wA + wB + wC) / ((wA + wB) * (wB + wC) * (wC + wA))
    expected = c9 * (1 + 3 * ca * cb * cc) / (rab * rac * rbc) ** 3
    e, _, ctx = gpu_state(system, pos)
    assert e == pytest.approx(expected, rel=ATM_E_TOL)
    f.setScaleFactor(0.7)
    f.updateParametersInContext(ctx)
    assert ctx.getState().getPotentialEnergy() == pytest.approx(0.7 * expected, rel=ATM_E_TOL)


def test_atm_centroid_sites():
    rng = np.random.default_rng(3)
    system = System()
    f = InteraxThreeBodyForce()
    pos = []
    for i in range(4):
        parts = []
        centre = np.array([0.4 * math.cos(2 * math.pi * i / 4), 0.4 * math.sin(2 * math.pi * i / 4), 0.1 * i])
        for j in range(i + 1):
            parts.append(system.addParticle(1.0))
            pos.append(centre + (rng.random(3) - 0.5) * 0.15)
        f.addSite(parts, 0.004 + 0.001 * i, 900.0 - 50 * i)
    system.addForce(f)
    compare(system, np.array(pos), energy_tol=ATM_E_TOL, force_tol=1e-5, scale="abs")


def test_atm_molecules_and_cutoff():
    system, f = single_sites(5)
    for i, m in enumerate([0, 0, -1, 3, -1]):
        p = f.getSiteParameters(i)
        f.setSiteParameters(i, p[0], p[1], p[2], p[3], m, p[5])
    pos = np.array([[0, 0, 0], [0.15, 0, 0], [0, 0.4, 0], [0.3, 0.3, 0.2], [-0.2, 0.1, 0.35]])
    compare(system, pos, energy_tol=ATM_E_TOL, force_tol=1e-5, scale="abs")
    system, f = single_sites(4)
    f.setCutoffDistance(0.5)
    pos = np.array([[0, 0, 0], [0.4, 0, 0], [0.2, 0.3, 0], [0.2, 0.75, 0]])
    e, frc, _, _, _ = compare(system, pos, energy_tol=ATM_E_TOL, force_tol=1e-5, scale="abs")
    assert np.all(frc[3] == 0.0)


@pytest.mark.parametrize("box_size", [3.5, 2.2])
def test_atm_periodic(box_size):
    """Cutoff 1.2 in boxes of 3.5 and 2.2 nm: the minimum images of a triple need not close."""
    rng = np.random.default_rng(4)
    system, f = single_sites(40)
    for i in range(40):
        p = f.getSiteParameters(i)
        f.setSiteParameters(i, p[0], p[1], p[2], p[3], i // 2, p[5])
    f.setCutoffDistance(1.2)
    f.setUsesPeriodicBoundaryConditions(True)
    box = np.diag([box_size] * 3)
    pos = []
    while len(pos) < 40:
        p = rng.random(3) * box_size * 3 - box_size
        ok = True
        for q in pos:
            d = p - q
            d -= box_size * np.floor(d / box_size + 0.5)
            ok &= d @ d > 0.25 ** 2
        if ok:
            pos.append(p)
    compare(system, np.array(pos), box, energy_tol=ATM_E_TOL, force_tol=1e-5, scale="abs")


@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("radius", [0.0, 0.3])
def test_atm_damping(method, radius):
    system, f = single_sites(4)
    f.setDampingMethod(method)
    f.setDampingScale(0.8)
    f.setCentroidDampingRadius(radius)
    pos = np.array([[0, 0, 0], [0.12, 0.02, 0], [0.05, 0.18, 0.03], [0.2, 0.2, 0.25]])
    compare(system, pos, energy_tol=ATM_E_TOL, force_tol=1e-5, scale="abs")


def test_atm_alchemical_and_overlap():
    system, f = single_sites(5)
    for i in (0, 1):
        p = f.getSiteParameters(i)
        f.setSiteParameters(i, p[0], p[1], p[2], p[3], p[4], True)
    f.setAlchemicalParameterName("lambda_test")
    pos = np.array([[0, 0, 0], [0.35, 0, 0], [0, 0.4, 0], [0.3, 0.3, 0.2], [-0.2, 0.1, 0.35]])
    ctx = Context(system)
    for lam in (1.0, 0.0, 0.25, 0.9):
        compare(system, pos, parameters={"lambda_test": lam}, context=ctx, energy_tol=ATM_E_TOL, force_tol=1e-5, scale="abs")
    # alchemical sites at lambda = 0 coinciding with another site: exactly zero, finite forces
    system, f = single_sites(5)
    for i in (0, 1):
        p = f.getSiteParameters(i)
        f.setSiteParameters(i, p[0], p[1], p[2], p[3], p[4], True)
    pos = np.array([[0, 0.4, 1e-9], [0.35, 0, 0], [0, 0.4, 0], [0.3, 0.3, 0.2], [-0.2, 0.1, 0.35]])
    e, frc, _ = gpu_state(system, pos, parameters={"lambda_sterics": 0.0})
    e_ref, _ = pyoracle.evaluate(system, pos, parameters={"lambda_sterics": 0.0})
    assert e == pytest.approx(e_ref, rel=ATM_E_TOL)
    assert np.all(np.isfinite(frc)) and np.all(frc[:2] == 0.0)


def test_atm_large_system():
    rng = np.random.default_rng(6)
    box_size = 2.4
    box = np.diag([box_size] * 3)
    centres = []
    while len(centres) < 50:
        p = rng.random(3) * box_size
        ok = True
        for q in centres:
            d = p - q
            d -= box_size * np.floor(d / box_size + 0.5)
            ok &= d @ d > 0.3 ** 2
        if ok:
            centres.append(p)
    system = System()
    system.setDefaultPeriodicBoxVectors(*box)
    f = InteraxThreeBodyForce()
    f.setCutoffDistance(1.0)
    f.setUsesPeriodicBoundaryConditions(True)
    f.setCentroidDampingRadius(0.25)
    f.setScaleFactor(1.3)
    pos = []
    for i in range(50):
        parts = []
        for j in range(3):
            parts.append(system.addParticle(1.0))
            pos.append(centres[i] + (rng.random(3) - 0.5) * 0.1)
        f.addSite(parts, 0.003 + 0.002 * (i % 3), 800.0 + 150 * (i % 4), 0.03, i, i < 3)
    system.addForce(f)
    compare(system, np.array(pos), box, {"lambda_sterics": 0.6}, scale="abs")


def test_atm_illegal_settings():
    system, f = single_sites(3)
    f.addSite([], 0.004, 900.0)
    with pytest.raises(OpenMMException, match="at least one particle"):
        Context(system)
    system, f = single_sites(3)
    f.addSite([3], 0.004, 900.0)
    with pytest.raises(OpenMMException, match="Illegal particle index for a site"):
        Context(system)
    system, f = single_sites(3)
    f.setDampingMethod(1)
    f.setSiteParameters(2, [2], 0.004, 900.0, 0.0, -1, False)
    with pytest.raises(OpenMMException, match="positive width"):
        Context(system)
    system, f = single_sites(3)
    f.setCutoffDistance(0.0)
    with pytest.raises(OpenMMException, match="cutoff distance must be positive"):
        Context(system)


# ------------------------------------------------------------------------------------------------------------------
# benchmark-shaped water systems
# ------------------------------------------------------------------------------------------------------------------
def test_water_small_box():
    cfg = W.CONFIGS["small"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=1,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    compare(system, pos, box)


def test_water_cluster_no_cutoff():
    system, pos, _ = W.water_cluster(32, seed=7)
    compare(system, pos)


@pytest.mark.slow
def test_water_24k_box():
    """The full-size plain configuration: 24,000 atoms, 8,000 sites, against the oracle."""
    cfg = W.CONFIGS["24k"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=1,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    e, f, e_ref, f_ref, ctx = compare(system, pos, box)
    pairs, triples = ctx.getCounts()
    cnt = []
    pyoracle.pair_force(0, system.getForce(0), pos, box, counts=cnt)
    c3 = []
    pyoracle.three_body(system.getForce(3), pos, box, counts=c3)
    assert pairs == cnt[0] and triples == c3[0]


def test_atm_lists_longer_than_staging():
    """A 300-water cluster without cutoffs: every site has up to 299 later sites, more than one staging of the wide
    triple kernel holds, so the (B, C) pairs are taken chunk by chunk."""
    system, pos, _ = W.water_cluster(300, seed=3)
    e, f, e_ref, f_ref, ctx = compare(system, pos, scale="abs")
    cnt = []
    pyoracle.three_body(system.getForce(3), pos, np.eye(3) * 10.0, counts=cnt)   # non-periodic: box unused
    assert ctx.getCounts()[1] == cnt[0]


def test_deterministic():
    """Fixed-point accumulation: two evaluations of the same input are bitwise identical."""
    cfg = W.CONFIGS["small"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=3,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    ctx = Context(system)
    ctx.setPositions(pos)
    a = ctx.getState()
    ctx2 = Context(system)
    ctx2.setPositions(pos)
    b = ctx2.getState()
    assert a.getPotentialEnergy() == b.getPotentialEnergy()
    assert np.array_equal(a.getForces(), b.getForces())


def test_graphs_match_direct_launches():
    """Evaluations and MD steps replayed from CUDA graphs equal direct launches bitwise, also after a parameter,
    the box and the positions change between replays (each change must invalidate the captured graph)."""
    cfg = W.CONFIGS["small"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=5,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    for f in range(3):
        fc = system.getForce(f)
        for i in range(0, system.getNumParticles(), 7):
            fc.setParticleParameters(i, *tuple(fc.getParticleParameters(i))[:-1], True)
    rng = np.random.default_rng(1)
    ctxs = [Context(system), Context(system)]
    ctxs[1]._check(ctxs[1]._lib.ix_set_graphs(ctxs[1]._ctx, 0))
    box2 = np.asarray(box) * 1.01
    steps = [(pos, box, 1.0), (pos + rng.normal(scale=0.01, size=pos.shape), box, 1.0),
             (pos, box, 0.4), (pos, box2, 0.4), (pos + rng.normal(scale=0.05, size=pos.shape), box2, 0.7)]
    for p, b, lam in steps:
        states = []
        for ctx in ctxs:
            ctx.setPeriodicBoxVectors(*np.asarray(b))
            ctx.setPositions(p)
            ctx.setParameter("lambda_sterics", lam)
            states.append(ctx.getState())
        assert states[0].getPotentialEnergy() == states[1].getPotentialEnergy()
        assert np.array_equal(states[0].getForces(), states[1].getForces())
    # kernel timing (events in the graph or on the streams; level 2 serialises the three-body chain): same results
    reference = states[0]
    for ctx in ctxs:
        ctx._check(ctx._lib.ix_set_profiling(ctx._ctx, 2))
        st = ctx.getState()
        assert st.getPotentialEnergy() == reference.getPotentialEnergy()
        assert np.array_equal(st.getForces(), reference.getForces())
        pair_ms, atm_ms = ctypes.c_double(), ctypes.c_double()
        ctx._check(ctx._lib.ix_get_kernel_times(ctx._ctx, ctypes.byref(pair_ms), ctypes.byref(atm_ms)))
        assert pair_ms.value > 0 and atm_ms.value > 0
        ctx._check(ctx._lib.ix_set_profiling(ctx._ctx, 0))
    vel = W.initial_velocities(system, 300.0, seed=2)
    runs = []
    for ctx in ctxs:
        ctx.setPeriodicBoxVectors(*np.asarray(box))
        ctx.setPositions(pos)
        runs.append(ctx.runVelocityVerlet(25, 0.001, vel))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    assert runs[0][2] == runs[1][2]


def test_neighbor_list_follows_motion():
    """Moving the particles by more than the skin forces a rebuild; the result stays exact."""
    cfg = W.CONFIGS["small"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=4,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    ctx = Context(system)
    rng = np.random.default_rng(0)
    for step in range(4):
        moved = pos + rng.normal(scale=0.03 * step, size=pos.shape)
        compare(system, moved, box, context=ctx, scale="abs")


def test_distinct_parameters_take_the_per_particle_path():
    """32 variants of each atom type perturbed within 1% (64 classes, beyond the 16 classes of the coefficient
    tables): the general pair kernel, against the oracle at the target bar."""
    system, pos, box = W.water_box(216, 1.865, 0.9, seed=17, three_body_cutoff=0.6, distinct=32)
    assert len({tuple(system.getForce(0).getParticleParameters(i)) for i in range(system.getNumParticles())}) > 16
    compare(system, pos, box)
