"""Fix the algorithmic work per interacting pair and per interacting triple by running the oracle on counting values.

TEST INFRASTRUCTURE: a one-time derivation whose result bench.py uses as a constant (F_PAIR, F_TRIPLE).

Counted operations: +, -, *, / and negation as one operation each, exp, sqrt and pow as one each; only the branch the
reference takes is counted (Taylor or closed form of the overlap, series or closed form of the damping).  The pair
count is the sum over the three pair terms of each term's own function, plus the pair driver once per pair (the three
terms share the geometry, cutoff test and force accumulation in one pass).  The triple count includes C9 and the three
displacements.

Run:  python oracle/count_ops.py        (the 24,000-atom water box, seed 1; ~1 minute)
"""
import ctypes
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path[:0] = [str(HERE), str(HERE.parent / "openmm-interax-plugin_b200")]

import pyoracle  # noqa: E402
from interaxplugin import workloads as W  # noqa: E402


def pair_ops(system, pos, box):
    L = pyoracle.lib()
    P = ctypes.c_void_p
    L.ox_pair_ops.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P, P, ctypes.c_double, ctypes.c_int,
                              ctypes.c_double, P]
    L.ox_pair_driver_ops.argtypes = [P]
    total = np.zeros(2)
    pairs = None
    for t in range(3):
        f = system.getForce(t)
        ex = np.ascontiguousarray(f._exclusion_array(), dtype=np.int32)
        s = pyoracle._PairSettings(f.getNonbondedMethod(), f.getCutoffDistance(), int(f.getUseSwitchingFunction()),
                                   f.getSwitchingDistance(), f.getSoftcoreRadius(), len(ex), pyoracle._ptr(ex))
        out = np.zeros(3)
        damping = f.getDampingScale() if t == 0 else 1.0
        om = f.getOverlapMethod() if t else 0
        L.ox_pair_ops(t, len(pos), pyoracle._ptr(np.ascontiguousarray(pos)),
                      pyoracle._ptr(np.ascontiguousarray(np.asarray(box, dtype=np.float64).reshape(9))),
                      ctypes.byref(s), pyoracle._ptr(np.ascontiguousarray(f._params_array())),
                      pyoracle._ptr(np.ascontiguousarray(f._alch_array())), damping, om, 1.0, pyoracle._ptr(out))
        total += out[:2]
        pairs = out[2]
    driver = np.zeros(2)
    L.ox_pair_driver_ops(pyoracle._ptr(driver))
    per_pair = total / pairs + driver
    return per_pair, pairs


def triple_ops(system, pos, box):
    L = pyoracle.lib()
    P = ctypes.c_void_p
    L.ox_three_body_ops.argtypes = [ctypes.c_int, P, P, ctypes.c_int, P, P, P, P, P, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_double, P]
    f = system.getForce(3)
    off, part, params, mol, alch = f._site_arrays()
    out = np.zeros(3)
    c = np.ascontiguousarray
    L.ox_three_body_ops(len(pos), pyoracle._ptr(c(pos)), pyoracle._ptr(c(np.asarray(box, dtype=np.float64).reshape(9))),
                        f.getNumSites(), pyoracle._ptr(c(off)), pyoracle._ptr(c(part)), pyoracle._ptr(c(params)),
                        pyoracle._ptr(c(mol)), pyoracle._ptr(c(alch)), f.getCutoffDistance(), f.getScaleFactor(),
                        f.getDampingMethod(), f.getDampingScale(), f.getCentroidDampingRadius(),
                        int(f.usesPeriodicBoundaryConditions()), 1.0, pyoracle._ptr(out))
    return out[:2] / out[2], out[2]


if __name__ == "__main__":
    cfg = W.CONFIGS["24k"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=1,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    (pa, pt), pairs = pair_ops(system, pos, box)
    (ta, tt), triples = triple_ops(system, pos, box)
    print(f"pairs {int(pairs)}: {pa:.2f} arithmetic + {pt:.2f} transcendental = F_PAIR {pa + pt:.1f} per pair")
    print(f"triples {int(triples)}: {ta:.2f} arithmetic + {tt:.2f} transcendental = F_TRIPLE {ta + tt:.1f} per triple")
