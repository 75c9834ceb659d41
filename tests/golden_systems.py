"""Build interaxplugin Systems from the committed golden fixtures (tests/golden/*.npz, written by make_golden.py)."""
from pathlib import Path

import numpy as np

from interaxplugin import (System, InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                           InteraxThreeBodyForce)

TERM_NAMES = ["dispersion", "exchange", "short_range", "three_body"]
GOLDEN = Path(__file__).resolve().parent / "golden"


def _pair_common(f, g, pre):
    f.setNonbondedMethod(int(g[pre + "method"]))
    f.setCutoffDistance(float(g[pre + "cutoff"]))
    f.setUseSwitchingFunction(bool(g[pre + "use_switch"]))
    f.setSwitchingDistance(float(g[pre + "switch_distance"]))
    f.setSoftcoreRadius(float(g[pre + "softcore_radius"]))
    f.setForceGroup(int(g[pre + "group"]))
    for p1, p2 in g[pre + "exclusions"]:
        f.addExclusion(int(p1), int(p2))


def load_golden(name):
    g = np.load(GOLDEN / f"{name}.npz")
    pos = g["positions"]
    box = g["box"]
    n = len(pos)
    system = System()
    for _ in range(n):
        system.addParticle(1.0)
    system.setDefaultPeriodicBoxVectors(*box)
    d = InteraxDispersionForce()
    for p, a in zip(g["disp_params"], g["disp_alch"]):
        d.addParticle(*p, isAlchemical=bool(a))
    d.setDampingScale(float(g["disp_damping_scale"]))
    d.setUseLongRangeCorrection(bool(g["disp_use_lrc"]))
    _pair_common(d, g, "disp_")
    system.addForce(d)
    x = InteraxExchangeForce()
    for p, a in zip(g["exch_params"], g["exch_alch"]):
        x.addParticle(*p, isAlchemical=bool(a))
    x.setOverlapMethod(int(g["exch_overlap_method"]))
    _pair_common(x, g, "exch_")
    system.addForce(x)
    s = InteraxShortRangeForce()
    for p, a in zip(g["sr_params"], g["sr_alch"]):
        s.addParticle(*p, isAlchemical=bool(a))
    s.setOverlapMethod(int(g["sr_overlap_method"]))
    _pair_common(s, g, "sr_")
    system.addForce(s)
    t = InteraxThreeBodyForce()
    off, part = g["atm_offsets"], g["atm_particles"]
    for i in range(len(g["atm_params"])):
        a, w, wd = g["atm_params"][i]
        t.addSite(part[off[i]:off[i + 1]].tolist(), a, w, wd, int(g["atm_molecule"][i]), bool(g["atm_alch"][i]))
    t.setCutoffDistance(float(g["atm_cutoff"]))
    t.setScaleFactor(float(g["atm_scale"]))
    t.setDampingMethod(int(g["atm_damping_method"]))
    t.setDampingScale(float(g["atm_damping_scale"]))
    t.setCentroidDampingRadius(float(g["atm_centroid_radius"]))
    t.setUsesPeriodicBoundaryConditions(bool(g["atm_periodic"]))
    t.setForceGroup(int(g["atm_group"]))
    system.addForce(t)
    expected = {term: (float(g["expected_energy_" + term]), g["expected_forces_" + term]) for term in TERM_NAMES}
    return system, pos, box, expected
