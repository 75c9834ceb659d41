"""Pin the FP64 oracle to the reference's own known answers.

* The export values of tests/data (tests/TestInteraxExportValues.h:150-197): per-term energies and forces of two
  systems computed by InteraxFF's export on OpenMM's Reference platform in double precision.  Tolerances as the
  reference's double-precision test: InteraxOrder2 within 1e-8 energy / 1e-7 x RMS force, Exact within 1e-6 / 1e-5.
* The closed-form and mpmath values of tests/TestInteraxExchangeForce.h:86-131 and the hand-computed dispersion
  coefficients of tests/TestInteraxDispersionForce.h:89-111.
"""
import math

import numpy as np
import pytest

import pyoracle
from golden_systems import load_golden, TERM_NAMES


@pytest.mark.parametrize("name", ["cluster", "methanol_box"])
@pytest.mark.parametrize("exact", [False, True])
def test_export_values(name, exact):
    system, positions, box, expected = load_golden(name)
    if exact:
        for f in system._forces:
            if hasattr(f, "setOverlapMethod"):
                f.setOverlapMethod(0)
    e_tol, f_tol = (1e-6, 1e-5) if exact else (1e-8, 1e-7)
    for group, term in enumerate(TERM_NAMES):
        e, f = pyoracle.evaluate(system, positions, box, groups=1 << group)
        E, F = expected[term]
        rms = math.sqrt((F ** 2).sum() / F.size)
        assert abs(e - E) <= e_tol * abs(E), (term, e, E)
        assert np.abs(f - F).max() <= f_tol * rms, term


def test_taylor_table_is_the_expansion_of_the_closed_form():
    """The derived coefficients: equal widths give exp(-x)(1 + x + x^2/3)/(64 pi), and the order-6 expansion
    reproduces the long-double closed form for small t."""
    value, deriv = pyoracle.taylor_table()
    assert value[0][:3] == pytest.approx([1 / 64, 1 / 64, 1 / 192], rel=1e-14)
    assert value[1][:4] == pytest.approx([-3 / 128, -3 / 128, -1 / 192, 1 / 384], rel=1e-13)
    for n in range(7):
        for k in range(9):
            nxt = (k + 1) * value[n][k + 1] if k + 1 < 9 else 0.0
            assert deriv[n][k] == pytest.approx(nxt - value[n][k], rel=1e-12, abs=1e-18)


def _overlap_ld(r, a, b):
    """Closed form in long double-ish precision via Python floats of numpy longdouble."""
    r, a, b = np.longdouble(r), np.longdouble(a), np.longdouble(b)
    d = b * b - a * a
    ea, eb = np.exp(-r / a), np.exp(-r / b)
    f = 4 * a * a * b * b / d ** 3 * (ea - eb) + r / d ** 2 * (a * ea + b * eb)
    return float(f / (8 * np.longdouble(math.pi) * r))


def test_overlap_known_answers():
    # mpmath value of tests/TestInteraxExchangeForce.h:102
    s, _ = pyoracle.slater_overlap(0.01, 0.02, 0.02 * (1 + 0.0002), 0)
    assert s == pytest.approx(5371.8136182115909371938804306761 / 9, rel=1e-12)
    # equal widths, tests/TestInteraxExchangeForce.h:110-131
    for r in (0.02, 0.1, 0.3):
        x = r / 0.025
        s, ds = pyoracle.slater_overlap(r, 0.025, 0.025, 0)
        assert s == pytest.approx(math.exp(-x) * (1 + x + x * x / 3) / (64 * math.pi * 0.025 ** 3), rel=1e-12)
        assert ds == pytest.approx(-math.exp(-x) * x * (1 + x) / 3 / (64 * math.pi * 0.025 ** 4), rel=1e-11)
    # closed form for well separated widths (no cancellation)
    for r, a, b in [(0.1, 0.02, 0.025), (0.15, 0.0198, 0.0276), (0.01, 0.018, 0.031)]:
        assert pyoracle.slater_overlap(r, a, b, 0)[0] == pytest.approx(_overlap_ld(r, a, b), rel=1e-12)
        assert pyoracle.slater_overlap(r, b, a, 0)[0] == pytest.approx(_overlap_ld(r, a, b), rel=1e-12)


def test_dispersion_coefficients():
    """tests/TestInteraxDispersionForce.h:89-111: at r = 2 nm the damping is 1 and E = -(C6/r^6+C8/r^8+C10/r^10)."""
    from interaxplugin import InteraxDispersionForce, System
    system = System()
    for _ in range(2):
        system.addParticle(1.0)
    f = InteraxDispersionForce()
    f.addParticle(2.0, 0.1, 0.005, 0.002, 0.025)
    f.addParticle(0.5, 0.01, 0.0002, 0.0003, 0.02)
    system.addForce(f)
    r = 2.0
    pos = np.array([[0, 0, 0], [0, 0, r]], dtype=float)
    e, forces = pyoracle.evaluate(system, pos)
    d = 0.002 * 0.5 + 0.0003 * 2.0
    c6 = 0.002 * 0.0003 * 2.0 * 0.5 / d
    c8 = 1.5 * 0.002 * 0.0003 * (2.0 * 0.01 + 0.1 * 0.5) / d
    c10 = (2 * 0.002 * 0.0003 * (2.0 * 0.0002 + 0.005 * 0.5) + 4.2 * 0.002 * 0.0003 * 0.1 * 0.01) / d
    assert e == pytest.approx(-(c6 / r ** 6 + c8 / r ** 8 + c10 / r ** 10), rel=1e-12)
    dedr = 6 * c6 / r ** 7 + 8 * c8 / r ** 9 + 10 * c10 / r ** 11
    assert forces[1][2] == pytest.approx(-dedr, rel=1e-12)


def test_tang_toennies_both_sides_of_the_switch():
    """f_n by the series below (n+1)/2 and the closed form above agree with a direct high-precision sum."""
    from mpmath import mp, mpf, exp, factorial
    mp.dps = 40
    for x in (0.01, 0.5, 2.0, 3.49, 3.51, 4.49, 4.51, 5.49, 5.51, 8.0, 20.0):
        f, df = pyoracle.tang_toennies(x)
        for i, n in enumerate((6, 8, 10)):
            exact = 1 - exp(-mpf(x)) * sum(mpf(x) ** k / factorial(k) for k in range(n + 1))
            assert f[i] == pytest.approx(float(exact), rel=1e-9, abs=1e-300)
