"""The restatement of the reference's CPU platform (oracle/cpu_platform.cpp), the timed CPU baseline, against the FP64
oracle: single-precision pair terms, so energies within 1e-5 of the sum of |energies| and forces within 1e-4 RMS
(the reference's single-precision tolerances, tests/TestInteraxPairForce.h:727-730), the same interacting pairs and
triples, and the same result on 1 and several threads up to the order of summation."""
import numpy as np
import pytest

import pyoracle
from interaxplugin import workloads as W
from parity import errors


def _check(system, pos, box, parameters=None, threads=3):
    absE = []
    e_ref, f_ref = pyoracle.evaluate(system, pos, box, parameters, abs_energy=absE)
    cpu = pyoracle.CpuPlatform(system, threads=threads)
    counts = []
    e, f = cpu.evaluate(pos, box, parameters, counts=counts)
    e_err, f_err = errors(e, f, e_ref, f_ref, max(absE[0], abs(e_ref)))
    assert e_err <= 1e-5 and f_err <= 1e-4, (e_err, f_err)
    ref_counts = []
    pyoracle.pair_force(0, system.getForce(0), pos, box if box is not None else np.eye(3), counts=ref_counts)
    assert counts[0] == ref_counts[0]
    e1, f1 = pyoracle.CpuPlatform(system, threads=1).evaluate(pos, box, parameters)
    assert abs(e1 - e) <= 1e-9 * max(absE[0], 1.0) and np.abs(f1 - f).max() <= 1e-3 * np.abs(f_ref).max()
    return counts


@pytest.mark.parametrize("seed", [1, 2])
def test_water_box(seed):
    cfg = W.CONFIGS["small"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=seed,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    counts = _check(system, pos, box)
    cnt = []
    pyoracle.three_body(system.getForce(3), pos, box, counts=cnt)
    assert counts[1] == cnt[0]


def test_alchemical_soft_core_and_switch():
    system, pos, box = W.water_box(120, 1.6, 0.7, seed=4, three_body_cutoff=0.5, alchemical_waters=range(6),
                                   softcore_radius=0.15)
    for f in system._forces[:3]:
        f.setUseSwitchingFunction(True)
        f.setSwitchingDistance(0.6)
    _check(system, pos, box, {"lambda_sterics": 0.4})


def test_cluster_no_cutoff():
    system, pos, _ = W.water_cluster(40, seed=3)
    _check(system, pos, None)
