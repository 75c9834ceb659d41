"""Seeded synthetic systems with the shapes of the benchmark configurations.

The reference benchmarks InteraxFF systems built with openff/packmol and a trained model (tests/python/benchmark.py),
none of which exist offline, so rigid 3-site water stands in for them:

* geometry: O-H 0.09572 nm, H-O-H 104.52 deg, molecule centres on a jittered cubic lattice (jitter U(-0.05, 0.05)
  nm), orientations uniformly random; all intramolecular pairs excluded (the InteraxFF convention);
* dispersion per atom type (O, H): C6 log-uniform in [1e-4, 3e-3] kJ/mol nm^6, C8 = C6 U(0.01, 0.03) nm^2,
  C10 = C8 U(0.01, 0.03) nm^2, Tang-Toennies rate b U(30, 45)/nm; polarizabilities O 1.2e-3, H 3e-4 nm^3; the XDM
  moments are m1 = 2 C6/alpha, m2 = C8/(1.5 alpha), m3 = (C10 - 2.1 alpha m2^2/m1)/(2 alpha) (which reproduce the
  like-pair C6, C8, C10 exactly), width 1/b, damping scale 1;
* exchange and short range per type: Slater exponent zeta U(25, 45)/nm (width 1/zeta, shared by both forces),
  valence charge q U(-1, -0.1), A = sqrt(K_A) |q| with K_A = 1 kJ/mol nm^3, K = U(-1500, 1500) |q| and
  L = U(1e4, 8e4) |q| kJ/mol;
* three-body: one site per water on its oxygen, molecule = water index, frequency U(700, 1300) kJ/mol,
  C9 log-uniform in [1e-7, 1e-5] kJ/mol nm^9 and alpha = (16 C9/(9 w))^(1/3), no damping.
"""
import math

import numpy as np

from .forces import (System, InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                     InteraxThreeBodyForce)

OH = 0.09572
HOH = math.radians(104.52)
MASS = {"O": 15.99943, "H": 1.007947}
WATERS_PER_NM3 = 33.4277    # 1.0 g/cm^3


def _water_frame():
    """Atom offsets of a water in its own frame, centred on the oxygen."""
    h1 = np.array([OH, 0.0, 0.0])
    h2 = np.array([OH * math.cos(HOH), OH * math.sin(HOH), 0.0])
    return np.array([[0.0, 0.0, 0.0], h1, h2])


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def type_parameters(rng):
    """Per-type parameters of O and H, drawn as described in the module docstring."""
    params = {}
    k_a = 1.0
    for t, alpha in (("O", 1.2e-3), ("H", 3e-4)):
        while True:
            c6 = math.exp(rng.uniform(math.log(1e-4), math.log(3e-3)))
            c8 = c6 * rng.uniform(0.01, 0.03)
            c10 = c8 * rng.uniform(0.01, 0.03)
            m1 = 2 * c6 / alpha
            m2 = c8 / (1.5 * alpha)
            m3 = (c10 - 2.1 * alpha * m2 * m2 / m1) / (2 * alpha)
            if m3 > 0:
                break
        b = rng.uniform(30.0, 45.0)
        zeta = rng.uniform(25.0, 45.0)
        q = rng.uniform(-1.0, -0.1)
        params[t] = dict(m1=m1, m2=m2, m3=m3, alpha=alpha, disp_width=1.0 / b, width=1.0 / zeta,
                         amplitude=math.sqrt(k_a) * abs(q), k=rng.uniform(-1500.0, 1500.0) * abs(q),
                         l=rng.uniform(1e4, 8e4) * abs(q))
    return params


def lattice_waters(num_waters, box_length, rng, jitter=0.05):
    """Water positions (3 num_waters x 3) on a jittered cubic lattice filling a cubic box."""
    per_side = int(math.ceil(num_waters ** (1.0 / 3.0) - 1e-9))
    spacing = box_length / per_side
    sites = [(i, j, k) for i in range(per_side) for j in range(per_side) for k in range(per_side)]
    chosen = rng.permutation(len(sites))[:num_waters] if len(sites) > num_waters else np.arange(num_waters)
    chosen = np.sort(chosen)
    frame = _water_frame()
    pos = np.empty((3 * num_waters, 3))
    for w, idx in enumerate(chosen):
        i, j, k = sites[idx]
        centre = (np.array([i, j, k]) + 0.5) * spacing + rng.uniform(-jitter, jitter, 3)
        pos[3 * w:3 * w + 3] = centre + frame @ _random_rotation(rng).T
    return pos


def cluster_waters(num_waters, rng, min_dist=0.26):
    """Waters with random centres inside a sphere at liquid density (rejection sampling)."""
    radius = (3.0 * num_waters / (4.0 * math.pi * WATERS_PER_NM3)) ** (1.0 / 3.0)
    centres = []
    frame = _water_frame()
    tries = 0
    while len(centres) < num_waters:
        tries += 1
        p = rng.uniform(-radius, radius, 3)
        if p @ p > radius * radius:
            continue
        if tries > 20000:
            radius *= 1.05
            tries = 0
        if all(np.sum((p - c) ** 2) > min_dist * min_dist for c in centres):
            centres.append(p)
    pos = np.empty((3 * num_waters, 3))
    for w, c in enumerate(centres):
        pos[3 * w:3 * w + 3] = c + frame @ _random_rotation(rng).T
    return pos


def build_water_system(positions, params, rng, method, cutoff, box_length=None, three_body_cutoff=None,
                       three_body=True, alchemical_waters=(), use_lrc=None, softcore_radius=0.0,
                       use_switch=False, switch_distance=-1.0, overlap_method=0, site_rng=None, rigid=False,
                       distinct=False):
    """A System of waters with the three pair forces and (optionally) the three-body force; rigid: each water's
    O-H, O-H and H-H distances constrained to the model geometry (the benchmark's rigid 3-site water); distinct: a
    number of variants of each atom type, every variant's parameters scaled by its own factors within 1%, and each
    water one variant (2 x distinct parameter classes, as in a system of many atom types: beyond the 16 classes of the
    kernels' per-class coefficient tables)."""
    num_waters = len(positions) // 3
    alch_set = set(int(w) for w in alchemical_waters)
    system = System()
    if box_length is not None:
        system.setDefaultPeriodicBoxVectors((box_length, 0, 0), (0, box_length, 0), (0, 0, box_length))
    disp, exch, sr = InteraxDispersionForce(), InteraxExchangeForce(), InteraxShortRangeForce()
    drng = np.random.default_rng(777)
    variants = {}
    if distinct:
        for t in ("O", "H"):
            variants[t] = []
            for _ in range(int(distinct)):
                f = 1.0 + 0.01 * drng.uniform(-1.0, 1.0, size=4)
                p = params[t]
                variants[t].append(dict(p, m1=p["m1"] * f[0], m2=p["m2"] * f[0], m3=p["m3"] * f[0],
                                        disp_width=p["disp_width"] * f[1], width=p["width"] * f[2],
                                        amplitude=p["amplitude"] * f[3], k=p["k"] * f[3], l=p["l"] * f[3]))
    for w in range(num_waters):
        alch = w in alch_set
        v = int(drng.integers(int(distinct))) if distinct else 0
        for t in ("O", "H", "H"):
            p = variants[t][v] if distinct else params[t]
            system.addParticle(MASS[t])
            disp.addParticle(p["m1"], p["m2"], p["m3"], p["alpha"], p["disp_width"], alch)
            exch.addParticle(p["amplitude"], p["width"], alch)
            sr.addParticle(p["k"], p["l"], p["width"], alch)
    if rigid:
        hh = 2.0 * OH * math.sin(HOH / 2.0)
        for w in range(num_waters):
            system.addConstraint(3 * w, 3 * w + 1, OH)
            system.addConstraint(3 * w, 3 * w + 2, OH)
            system.addConstraint(3 * w + 1, 3 * w + 2, hh)
    for f, group in ((disp, 0), (exch, 1), (sr, 2)):
        f.setNonbondedMethod(method)
        f.setCutoffDistance(cutoff)
        f.setForceGroup(group)
        f.setSoftcoreRadius(softcore_radius)
        f.setUseSwitchingFunction(use_switch)
        f.setSwitchingDistance(switch_distance)
        for w in range(num_waters):
            f.addExclusion(3 * w, 3 * w + 1)
            f.addExclusion(3 * w, 3 * w + 2)
            f.addExclusion(3 * w + 1, 3 * w + 2)
        system.addForce(f)
    disp.setDampingScale(1.0)
    disp.setUseLongRangeCorrection(method == InteraxDispersionForce.CutoffPeriodic if use_lrc is None else use_lrc)
    exch.setOverlapMethod(overlap_method)
    sr.setOverlapMethod(overlap_method)
    if three_body:
        srng = site_rng if site_rng is not None else rng
        atm = InteraxThreeBodyForce()
        for w in range(num_waters):
            omega = srng.uniform(700.0, 1300.0)
            c9 = math.exp(srng.uniform(math.log(1e-7), math.log(1e-5)))
            alpha = (16.0 * c9 / (9.0 * omega)) ** (1.0 / 3.0)
            atm.addSite([3 * w], alpha, omega, 0.0, w, w in alch_set)
        atm.setCutoffDistance(three_body_cutoff if three_body_cutoff is not None else 1.2)
        atm.setUsesPeriodicBoundaryConditions(box_length is not None)
        atm.setForceGroup(3)
        system.addForce(atm)
    return system


def water_box(num_waters, box_length, cutoff, seed=0, three_body_cutoff=None, three_body=True, **kw):
    """Periodic water box (configurations 0, 1 and 4 of the benchmark)."""
    rng = np.random.default_rng(seed)
    params = type_parameters(rng)
    pos = lattice_waters(num_waters, box_length, rng)
    system = build_water_system(pos, params, rng, InteraxDispersionForce.CutoffPeriodic, cutoff, box_length,
                                three_body_cutoff, three_body, **kw)
    return system, pos, np.diag([box_length] * 3)


def water_cluster(num_waters, seed=0, params=None, three_body=True):
    """Non-periodic water cluster with no cutoff (configuration 2 of the benchmark)."""
    rng = np.random.default_rng(seed)
    params = params or type_parameters(np.random.default_rng(12345))
    pos = cluster_waters(num_waters, rng)
    system = build_water_system(pos, params, rng, InteraxDispersionForce.NoCutoff, 1.0, None, 100.0, three_body,
                                use_lrc=False)
    return system, pos, None


def cluster_set(num_clusters, seed=1, stream=0):
    """The batched workload: num_clusters water clusters of 2..32 waters (configuration 2 of the benchmark), cluster k
    drawn from its own seed so that any subset can be rebuilt alone.  Returns (systems, positions)."""
    sizes = cluster_sizes(num_clusters, seed, stream)
    systems, positions = [], []
    for k in range(num_clusters):
        s, p = cluster_of_set(k, sizes, seed, stream)
        systems.append(s)
        positions.append(p)
    return systems, positions


def cluster_of_set(k, sizes, seed=1, stream=0):
    """Cluster k of cluster_set (sizes from cluster_sizes), built alone: (system, positions)."""
    s, p, _ = water_cluster(int(sizes[k]), seed=seed * 100003 + 7919 * stream + k)
    return s, p


def cluster_sizes(num_clusters, seed=1, stream=0):
    """The water counts of cluster_set's clusters, without building them."""
    return np.random.default_rng(seed + 7919 * stream).integers(2, 33, size=num_clusters)


def box_length_for(num_waters):
    return (num_waters / WATERS_PER_NM3) ** (1.0 / 3.0)


# The benchmark configurations (sizes as stated by the benchmark definition).
CONFIGS = {
    "small": dict(num_waters=216, box_length=1.865, cutoff=0.9, three_body_cutoff=0.6),
    "24k": dict(num_waters=8000, box_length=6.208, cutoff=1.0, three_body_cutoff=0.6),
    "96k": dict(num_waters=32000, box_length=9.855, cutoff=1.0, three_body_cutoff=0.8),
}


def initial_velocities(system, temperature, seed=0):
    """Maxwell-Boltzmann velocities (nm/ps) at `temperature` K, zero total momentum."""
    rng = np.random.default_rng(seed)
    kT = 0.00831446261815324 * temperature
    m = np.array([system.getParticleMass(i) for i in range(system.getNumParticles())])
    v = rng.normal(size=(len(m), 3)) * np.sqrt(kT / m)[:, None]
    v -= (m[:, None] * v).sum(0) / m.sum()
    return v
