"""Convert the reference plugin's export-value test data into compact fixtures.

The reference holds two systems with per-term energies and forces computed by the InteraxFF export on OpenMM's
Reference platform in double precision (tests/data/{cluster,methanol_box}/{system.xml,reference.txt}, read by
tests/TestInteraxExportValues.h:77-127).  This script reads them from a checkout of the reference and writes one .npz
per system with the positions, box, every force's settings and per-particle parameters, and the expected values.

Run:  python tests/golden/make_golden.py /path/to/openmm-interax-plugin
"""
import sys
import xml.etree.ElementTree as ET
from pathlib import Path

import numpy as np

TERMS = ["dispersion", "exchange", "short_range", "three_body"]


def read_reference(path):
    """reference.txt: box, positions, then 'term <name> <group> <energy>' followed by the forces."""
    lines = [l for l in Path(path).read_text().splitlines() if l and not l.startswith("#")]
    out = {"energies": {}, "forces": {}}
    i = 0
    while i < len(lines):
        words = lines[i].split()
        if words[0] == "box":
            out["periodic"] = words[1] != "none"
            out["box"] = np.array([float(w) for w in words[1:]]).reshape(3, 3) if out["periodic"] else np.eye(3) * 2.0
            i += 1
        elif words[0] == "positions":
            n = int(words[1])
            out["positions"] = np.array([[float(w) for w in lines[i + 1 + k].split()] for k in range(n)])
            i += 1 + n
        elif words[0] == "term":
            name, group, energy = words[1], int(words[2]), float(words[3])
            n = len(out["positions"])
            out["energies"][name] = (group, energy)
            out["forces"][name] = np.array([[float(w) for w in lines[i + 1 + k].split()] for k in range(n)])
            i += 1 + n
        else:
            raise ValueError(lines[i])
    return out


def pair_settings(force):
    a = force.attrib
    ex = [(int(e.attrib["p1"]), int(e.attrib["p2"])) for e in force.find("Exclusions")]
    return dict(method=int(a["method"]), cutoff=float(a["cutoff"]), use_switch=int(a["useSwitchingFunction"]),
                switch_distance=float(a["switchingDistance"]), softcore_radius=float(a["softcoreRadius"]),
                group=int(a["forceGroup"]), exclusions=np.array(ex, dtype=np.int32).reshape(-1, 2))


def main(ref_root):
    out_dir = Path(__file__).resolve().parent
    for name in ["cluster", "methanol_box"]:
        data = Path(ref_root) / "tests" / "data" / name
        ref = read_reference(data / "reference.txt")
        root = ET.parse(data / "system.xml").getroot()
        arrays = {"positions": ref["positions"], "box": ref["box"], "periodic": np.array(ref["periodic"])}
        for force in root.find("Forces"):
            kind = force.attrib["type"]
            parts = force.find("Particles")
            if kind == "InteraxDispersionForce":
                s = pair_settings(force)
                arrays["disp_params"] = np.array([[float(p.attrib[k]) for k in ("m1", "m2", "m3", "alpha", "width")]
                                                  for p in parts])
                arrays["disp_alch"] = np.array([int(p.attrib["alchemical"]) for p in parts], dtype=np.uint8)
                arrays["disp_damping_scale"] = np.array(float(force.attrib["dampingScale"]))
                arrays["disp_use_lrc"] = np.array(int(force.attrib["useLongRangeCorrection"]))
                for k, v in s.items():
                    arrays["disp_" + k] = np.array(v)
            elif kind in ("InteraxExchangeForce", "InteraxShortRangeForce"):
                pre = "exch_" if kind == "InteraxExchangeForce" else "sr_"
                keys = ("amplitude", "width") if pre == "exch_" else ("k", "l", "width")
                s = pair_settings(force)
                arrays[pre + "params"] = np.array([[float(p.attrib[k]) for k in keys] for p in parts])
                arrays[pre + "alch"] = np.array([int(p.attrib["alchemical"]) for p in parts], dtype=np.uint8)
                arrays[pre + "overlap_method"] = np.array(int(force.attrib["overlapMethod"]))
                for k, v in s.items():
                    arrays[pre + k] = np.array(v)
            elif kind == "InteraxThreeBodyForce":
                a = force.attrib
                sites = force.find("Sites")
                offsets, particles, params, molecule, alch = [0], [], [], [], []
                for site in sites:
                    particles += [int(p.attrib["index"]) for p in site]
                    offsets.append(len(particles))
                    params.append([float(site.attrib[k]) for k in ("alpha", "frequency", "width")])
                    molecule.append(int(site.attrib["molecule"]))
                    alch.append(int(site.attrib["alchemical"]))
                arrays.update(atm_offsets=np.array(offsets, dtype=np.int32),
                              atm_particles=np.array(particles, dtype=np.int32),
                              atm_params=np.array(params), atm_molecule=np.array(molecule, dtype=np.int32),
                              atm_alch=np.array(alch, dtype=np.uint8), atm_cutoff=np.array(float(a["cutoff"])),
                              atm_scale=np.array(float(a["scaleFactor"])),
                              atm_damping_method=np.array(int(a["dampingMethod"])),
                              atm_damping_scale=np.array(float(a["dampingScale"])),
                              atm_centroid_radius=np.array(float(a["centroidDampingRadius"])),
                              atm_periodic=np.array(int(a["usesPeriodic"])), atm_group=np.array(int(a["forceGroup"])))
        for term in TERMS:
            group, energy = ref["energies"][term]
            arrays["expected_energy_" + term] = np.array(energy)
            arrays["expected_group_" + term] = np.array(group)
            arrays["expected_forces_" + term] = ref["forces"][term]
        np.savez_compressed(out_dir / f"{name}.npz", **arrays)
        print(name, {k: v.shape for k, v in arrays.items() if v.ndim})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the reference project checkout>")
    main(sys.argv[1])
