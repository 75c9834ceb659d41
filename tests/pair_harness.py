"""The reference's pair-test harness restated, with a case of every option of a pair force: the checker of
test_oracle_pair_harness.py (the FP64 oracle) and test_gpu_harness.py (the B200 kernels).

The reference's tests (tests/TestInteraxPairForce.h:59-148) compute the expected energy of a pair force as a loop over
all pairs of particles: exclusions; periodic minimum images; the cutoff; for a pair with exactly one alchemical
particle the soft-core distance (r^6 + (1 - lambda) R^6)^(1/6) and the factor lambda; the switching function
1 - 10x^3 + 15x^4 - 6x^5; and the force of each pair as the five-point derivative of that pair energy along the pair.
The pair energies are the three forces' test models (tests/TestInteraxDispersionForce.h:63-78,
tests/TestInteraxExchangeForce.h:66-75, tests/TestInteraxShortRangeForce.h:66-76) over the Slater overlap of
normalized densities exp(-r/s)/(8 pi s^3).  Restated here in 40-digit arithmetic (mpmath), so that the overlap's
closed form, which cancels for nearly equal widths, and the Tang-Toennies sums need no series switches.
"""
import numpy as np
import pytest

from interaxplugin import (InteraxDispersionForce, InteraxExchangeForce, InteraxPairForce, InteraxShortRangeForce,
                           System)

mpmath = pytest.importorskip("mpmath")
mp = mpmath.mp


def overlap(r, a, b):
    """S(r; a, b), the overlap of two normalized Slater densities of widths a and b; the equal-width limit
    exp(-x) (1 + x + x^2/3)/(64 pi a^3), x = r/a, when a = b."""
    if a == b:
        x = r / a
        return mpmath.exp(-x) * (1 + x + x * x / 3) / (64 * mp.pi * a ** 3)
    d = b * b - a * a
    ea, eb = mpmath.exp(-r / a), mpmath.exp(-r / b)
    return (4 * a * a * b * b / d ** 3 * (ea - eb) + r / d ** 2 * (a * ea + b * eb)) / (8 * mp.pi * r)


def tang_toennies(n, x):
    """f_n(x) = 1 - exp(-x) sum_{k<=n} x^k/k!"""
    return 1 - mpmath.exp(-x) * sum(x ** k / mpmath.factorial(k) for k in range(n + 1))


def dispersion_pair(p, q, scale):
    """The dispersion model's pair energy function: C6, C8, C10 of the pair from (m1, m2, m3, alpha, width)."""
    m1i, m2i, m3i, ai, wi = (mpmath.mpf(v) for v in p)
    m1j, m2j, m3j, aj, wj = (mpmath.mpf(v) for v in q)
    if ai * aj == 0:
        return None
    den = ai * m1j + aj * m1i
    a2 = ai * aj
    c6 = a2 * m1i * m1j / den
    c8 = mpmath.mpf(1.5) * a2 * (m1i * m2j + m2i * m1j) / den
    c10 = (2 * a2 * (m1i * m3j + m3i * m1j) + mpmath.mpf("4.2") * a2 * m2i * m2j) / den

    def energy(r):
        x = mpmath.mpf(scale) * 2 * r / (wi + wj)
        return -(tang_toennies(6, x) * c6 / r ** 6 + tang_toennies(8, x) * c8 / r ** 8 +
                 tang_toennies(10, x) * c10 / r ** 10)
    return energy


def exchange_pair(p, q):
    """The exchange model: A_i A_j S(r)."""
    ai, wi = (mpmath.mpf(v) for v in p)
    aj, wj = (mpmath.mpf(v) for v in q)
    if wi * wj == 0:
        return None
    return lambda r: ai * aj * overlap(r, wi, wj)


def short_range_pair(p, q):
    """The short-range model: (K_i + K_j)/2 St + (L_i + L_j)/2 St^2, St = 8 pi (s_i + s_j)^3 S."""
    ki, li, wi = (mpmath.mpf(v) for v in p)
    kj, lj, wj = (mpmath.mpf(v) for v in q)
    if wi * wj == 0:
        return None

    def energy(r):
        st = 8 * mp.pi * (wi + wj) ** 3 * overlap(r, wi, wj)
        return (ki + kj) / 2 * st + (li + lj) / 2 * st * st
    return energy


def switching(r, start, cutoff):
    if r <= start:
        return mpmath.mpf(1)
    if r >= cutoff:
        return mpmath.mpf(0)
    x = (r - start) / (cutoff - start)
    return 1 - 10 * x ** 3 + 15 * x ** 4 - 6 * x ** 5


def minimum_image(d, box):
    """The shortest periodic image of d in a box whose rows are its (reduced) edge vectors: d reduced along c, b and a,
    then the nearest of it and its 26 neighbouring images."""
    for k in (2, 1, 0):
        d = d - box[k] * round(d[k] / box[k][k])
    images = [d + i * box[0] + j * box[1] + k * box[2] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)]
    return min(images, key=lambda v: v @ v)


def harness(force, model, positions, box, lam):
    """Energy, forces and the sum of |pair energies| before switching (the error scale) of a pair force, by the loop
    over all pairs, in 40-digit arithmetic."""
    with mpmath.workdps(40):
        return _harness(force, model, positions, box, lam)


def _harness(force, model, positions, box, lam):
    n = force.getNumParticles()
    excluded = {tuple(sorted(force.getExclusionParticles(k))) for k in range(force.getNumExclusions())}
    use_cutoff = force.getNonbondedMethod() != InteraxPairForce.NoCutoff
    periodic = force.getNonbondedMethod() == InteraxPairForce.CutoffPeriodic
    cutoff, start = mpmath.mpf(force.getCutoffDistance()), mpmath.mpf(force.getSwitchingDistance())
    radius, lam = mpmath.mpf(force.getSoftcoreRadius()), mpmath.mpf(lam)
    energy, abs_sum = mpmath.mpf(0), mpmath.mpf(0)
    forces = np.zeros((n, 3))
    for i in range(n):
        for j in range(i + 1, n):
            if (i, j) in excluded:
                continue
            d = positions[j] - positions[i]
            if periodic:
                d = minimum_image(d, box)
            r = mpmath.sqrt(sum(mpmath.mpf(float(v)) ** 2 for v in d))
            base = model(force.getParticleParameters(i)[:-1], force.getParticleParameters(j)[:-1])
            if base is None:
                continue
            alchemical_pair = force.getParticleIsAlchemical(i) != force.getParticleIsAlchemical(j)

            def pair_energy(s, switch=True):
                if use_cutoff and s >= cutoff:
                    return mpmath.mpf(0)
                s_eff = (s ** 6 + (1 - lam) * radius ** 6) ** (mpmath.mpf(1) / 6) if alchemical_pair else s
                e = base(s_eff)
                if use_cutoff and force.getUseSwitchingFunction() and switch:
                    e *= switching(s, start, cutoff)
                return e * lam if alchemical_pair else e

            e = pair_energy(r)
            if e == 0:
                continue
            energy += e
            abs_sum += abs(pair_energy(r, False))
            h = mpmath.mpf("1e-12")
            dedr = (pair_energy(r - 2 * h) - 8 * pair_energy(r - h) + 8 * pair_energy(r + h) -
                    pair_energy(r + 2 * h)) / (12 * h)
            f = d * float(dedr / r)
            forces[i] += f
            forces[j] -= f
    return float(energy), forces, float(abs_sum)


# exact, nearly equal (t = 0.015: the oracle's series branch) and distinct widths, so every overlap path is taken
WIDTHS = [0.020, 0.0203, 0.024, 0.024, 0.030, 0.020, 0.0203, 0.026, 0.024, 0.030, 0.022, 0.020, 0.0203, 0.024]
ALCHEMICAL = {3, 8, 12}
EXCLUSIONS = [(1, 2), (7, 13), (4, 10)]


def build(kind, method, rng):
    force = {"dispersion": InteraxDispersionForce, "exchange": InteraxExchangeForce,
             "short_range": InteraxShortRangeForce}[kind]()
    for i, w in enumerate(WIDTHS):
        alch = i in ALCHEMICAL
        if kind == "dispersion":
            # particle 9 has no polarizability (a lone pair): it interacts with nothing
            alpha = 0.0 if i == 9 else rng.uniform(5e-4, 2e-3)
            force.addParticle(rng.uniform(1.5, 3.5), rng.uniform(0.03, 0.08), rng.uniform(1e-3, 3e-3), alpha, w, alch)
        elif kind == "exchange":
            force.addParticle(rng.uniform(1.0, 10.0), w, alch)
        else:
            force.addParticle(rng.uniform(-1000.0, 1000.0), rng.uniform(1e4, 8e4), w, alch)
    for p, q in EXCLUSIONS:
        force.addExclusion(p, q)
    force.setNonbondedMethod(method)
    if method != InteraxPairForce.NoCutoff:
        force.setCutoffDistance(0.7)
        force.setUseSwitchingFunction(True)
        force.setSwitchingDistance(0.55)
    force.setSoftcoreRadius(0.12)
    if kind == "dispersion":
        force.setDampingScale(0.8)
    system = System()
    for _ in WIDTHS:
        system.addParticle(1.0)
    system.addForce(force)
    return system, force


MODELS = {"dispersion": lambda p, q: dispersion_pair(p, q, 0.8), "exchange": exchange_pair,
          "short_range": short_range_pair}


BOX_LENGTH = 1.5


def harness_positions(rng):
    """12 particles on a jittered 3 x 2 x 2 lattice of the rectangular box, and two more 0.12 and 0.15 nm from
    particles 0 and 5; the first of those is alchemical, so its pair with particle 0 is in the soft core."""
    grid = np.array([[x, y, z] for x in range(3) for y in range(2) for z in range(2)], dtype=float)
    pos = (grid + 0.5) * np.array([BOX_LENGTH / 3, BOX_LENGTH / 2, BOX_LENGTH / 2])
    pos += rng.uniform(-0.08, 0.08, pos.shape)
    return np.vstack([pos, pos[0] + [0.12, 0.0, 0.0], pos[5] + [0.0, 0.15, 0.0]])


# a triclinic box in reduced form (each edge's components along the earlier edges within half of them); its
# perpendicular widths (1.452, 1.461, 1.5 nm) stay above twice the 0.7 nm cutoff, so each pair has one image within it
TRICLINIC = np.array([[1.55, 0.0, 0.0], [0.4, 1.5, 0.0], [-0.3, 0.35, 1.5]])

KINDS = ["dispersion", "exchange", "short_range"]
# (nonbonded method, lambda, triclinic box): periodic with cutoff and switching in both boxes, and no cutoff
CASES = [(InteraxPairForce.CutoffPeriodic, 0.6, False), (InteraxPairForce.CutoffPeriodic, 0.6, True),
         (InteraxPairForce.NoCutoff, 0.3, False)]


def case_box(triclinic):
    return TRICLINIC if triclinic else np.eye(3) * BOX_LENGTH
