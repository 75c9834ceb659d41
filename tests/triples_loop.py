"""The reference three-body test's all-triples loop restated, with a periodic case of every option: the checker of
test_oracle_three_body.py (the FP64 oracle) and test_gpu_harness.py (the B200 kernels).

computeReferenceEnergy and computeReferenceForces (tests/TestInteraxThreeBodyForce.h:71-129 and the finite
differences after them): the energy as a loop over all triples of sites with the cosines of the angles at the
vertices, distinct molecules, the cutoff on all three sides, periodic minimum images, Tang-Toennies and centroid
damping and the alchemical factor; the forces as central differences of that energy.
"""
import itertools
import math

import numpy as np

from interaxplugin import InteraxThreeBodyForce, System

# the three site types of testTriple (tests/TestInteraxThreeBodyForce.h:185-222): alpha (nm^3), frequency (kJ/mol),
# width (nm)
SITE_TYPES = [(0.004087456746801944, 911.0681141195369, 0.03), (0.0016246535729804365, 1262.664320774599, 0.025),
              (0.008817709933796472, 747.5256543931184, 0.035)]


def c9_of(a, b, c):
    """C9 of three sites from their (alpha, frequency) (InteraxThreeBodyForceImpl.h:69-72)."""
    (aa, wa), (ab, wb), (ac, wc) = a, b, c
    return 1.5 * aa * ab * ac * wa * wb * wc * (wa + wb + wc) / ((wa + wb) * (wb + wc) * (wc + wa))


def single_sites(types):
    """A System of one single-particle site per (alpha, frequency, width)."""
    system = System()
    force = InteraxThreeBodyForce()
    for i, (a, w, s) in enumerate(types):
        system.addParticle(1.0)
        force.addSite([i], a, w, s)
    system.addForce(force)
    return system, force


def tang_toennies(n, x):
    """f_n(x) = 1 - exp(-x) sum_{k<=n} x^k/k!, summed as its tail exp(-x) sum_{k>n} x^k/k! below x = n + 1, where the
    closed form cancels."""
    term, partial = 1.0, 1.0
    for k in range(1, n + 1):
        term *= x / k
        partial += term
    if x >= n + 1:
        return 1.0 - math.exp(-x) * partial
    tail = 0.0
    for k in range(n + 1, 400):
        term *= x / k
        tail += term
        if term < 1e-30 * tail:
            break
    return math.exp(-x) * tail


def brute_force_energy(sites, positions, box_length, cutoff, scale, tt_scale, radius, lam):
    """The ATM energy as a loop over all triples of sites (the reference test's computeReferenceEnergy).  `sites`:
    (particles, alpha, frequency, width, molecule, alchemical) per site; a negative molecule is the site's own."""
    centre = [np.mean([positions[p] for p in s[0]], axis=0) for s in sites]
    molecule = [s[4] if s[4] >= 0 else -1 - i for i, s in enumerate(sites)]

    def delta(i, j):
        d = centre[j] - centre[i]
        return d - box_length * np.floor(d / box_length + 0.5)

    def damping(i, j, r):
        f = 1.0
        if tt_scale:
            f *= tang_toennies(3, tt_scale * 2 * r / (sites[i][3] + sites[j][3]))
        if radius > 0:
            f *= 1 - math.exp(-(r / radius) ** 6)
        return f

    energy = 0.0
    for i, j, k in itertools.combinations(range(len(sites)), 3):
        if molecule[i] == molecule[j] or molecule[i] == molecule[k] or molecule[j] == molecule[k]:
            continue
        a, b, c = delta(i, j), delta(i, k), delta(j, k)
        ra, rb, rc = np.linalg.norm(a), np.linalg.norm(b), np.linalg.norm(c)
        if ra >= cutoff or rb >= cutoff or rc >= cutoff:
            continue
        # the angle at each vertex lies between the vectors to its two neighbours
        cos_a, cos_b, cos_c = a @ b / (ra * rb), -(a @ c) / (ra * rc), b @ c / (rb * rc)
        c9 = scale * c9_of(sites[i][1:3], sites[j][1:3], sites[k][1:3])
        e = c9 * (1 + 3 * cos_a * cos_b * cos_c) / (ra * rb * rc) ** 3
        e *= damping(i, j, ra) * damping(i, k, rb) * damping(j, k, rc)
        if sites[i][5] or sites[j][5] or sites[k][5]:
            e *= lam
        energy += e
    return energy


BOX_LENGTH, CUTOFF, SCALE, LAMBDA = 1.3, 0.6, 0.8, 0.6
# damping scale and centroid radius where both dampings are of order one at the sites' distances (0.3-0.6 nm)
DAMPING_CASES = [(0.0, 0.0), (0.3, 0.0), (0.0, 0.4), (0.3, 0.4)]


def loop_case(tt_scale, radius, rng):
    """A periodic case of every option: the System, its force, the sites as the loop takes them, and positions."""
    box_length, cutoff = BOX_LENGTH, CUTOFF
    # 13 particles: 8 single-particle sites and 2 centroid sites of 2 and 3 particles; two sites share molecule 5, two
    # share molecule 2, two are alchemical
    layout = [[0], [1], [2], [3], [4], [5], [6], [7], [8, 9], [10, 11, 12]]
    molecules = [5, 5, -1, 2, -1, -1, 2, -1, -1, -1]
    alchemical = [False, False, True, False, False, False, False, True, False, False]
    for attempt in range(100):
        # one site per cell of a jittered 3 x 3 x 3 grid cut to 10 sites, its particles within 0.05 nm of the site
        cells = rng.permutation(27)[:10]
        pos = np.zeros((13, 3))
        for s, parts in enumerate(layout):
            grid = np.array([cells[s] % 3, (cells[s] // 3) % 3, cells[s] // 9], dtype=float)
            site = (grid + 0.5 + rng.uniform(-0.2, 0.2, 3)) * box_length / 3
            for p in parts:
                pos[p] = site + rng.uniform(-0.05, 0.05, 3)
        # no side within 2e-3 nm of the cutoff, so that the central differences do not straddle it
        centres = np.array([pos[parts].mean(0) for parts in layout])
        d = centres[:, None] - centres[None]
        d -= box_length * np.floor(d / box_length + 0.5)
        r = np.linalg.norm(d, axis=-1)
        if np.all(np.abs(r - cutoff) > 2e-3):
            break
    system = System()
    force = InteraxThreeBodyForce()
    for _ in range(13):
        system.addParticle(1.0)
    sites = []
    for s, parts in enumerate(layout):
        a, w, width = SITE_TYPES[s % 3]
        force.addSite(parts, a, w, width, molecules[s], alchemical[s])
        sites.append((parts, a, w, width, molecules[s], alchemical[s]))
    force.setCutoffDistance(cutoff)
    force.setUsesPeriodicBoundaryConditions(True)
    force.setScaleFactor(SCALE)
    if tt_scale:
        force.setDampingMethod(InteraxThreeBodyForce.TangToennies)
        force.setDampingScale(tt_scale)
    force.setCentroidDampingRadius(radius)
    system.addForce(force)
    return system, force, sites, pos


def loop_energy_and_forces(sites, pos, tt_scale, radius, lam=LAMBDA):
    """The loop's energy, and the forces as five-point central differences of it."""
    def energy(x):
        return brute_force_energy(sites, x, BOX_LENGTH, CUTOFF, SCALE, tt_scale, radius, lam)

    h = 1e-5
    fd = np.zeros_like(pos)
    for p in range(len(pos)):
        for k in range(3):
            def shifted(t):
                x = pos.copy()
                x[p, k] += t
                return energy(x)
            fd[p, k] = -(shifted(-2 * h) - 8 * shifted(-h) + 8 * shifted(h) - shifted(2 * h)) / (12 * h)
    return energy(pos), fd
