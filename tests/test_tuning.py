"""The autotuner's plumbing on the host: the constants it searches are exactly the IX_TUNE_* macros of
csrc/ix_tuning.h, its candidates stay within what the kernels accept, and the build turns tuning.json into compiler
definitions."""
import json
import re
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "openmm-interax-plugin_b200"
sys.path.insert(0, str(PKG))

import build_lib  # noqa: E402
import tune  # noqa: E402


def header_macros():
    text = (PKG / "csrc" / "ix_tuning.h").read_text()
    return dict(re.findall(r"#define (IX_TUNE_\w+) (\S+)", text))


def test_tuner_covers_every_macro_with_the_header_defaults():
    macros = header_macros()
    assert set(tune.DEFAULTS) == set(macros)
    for name, value in tune.DEFAULTS.items():
        assert float(macros[name].rstrip("f")) == float(value), name
    for _, options in tune.GROUPS:
        for o in options:
            assert set(o) <= set(macros)


def test_candidates_respect_the_kernels_limits():
    for _, options in tune.GROUPS:
        for o in options:
            v = dict(tune.DEFAULTS, **o)
            # the fast triple kernel gathers at most two staged neighbors per lane
            assert v["IX_TUNE_ATM_FAST"] in (32, 64)
            assert v["IX_TUNE_PAIR_ROUND"] % 32 == 0 and v["IX_TUNE_ATM_ROUND"] % 32 == 0
            # per-block static shared memory of the pair kernel stays within 48 KB
            per_warp = 1024 + 1024 + 256 + 384 + 2048 + 16 * v["IX_TUNE_PAIR_ROUND"] + \
                (2048 if v["IX_TUNE_PAIR_COLUMN_LISTS"] else 2)
            assert per_warp * v["IX_TUNE_PAIR_WARPS"] <= 48 * 1024
            # the fast triple kernel's 4 warps: staged neighbors (two float4 and an int each) and a round's B and C
            # forces, within 48 KB of static shared memory, and the blocks per SM it asks for within 228 KB
            rounds = 1 if v["IX_TUNE_ATM_ACCUM"] else v["IX_TUNE_ATM_ROUND"]
            sums = 3 * 8 * v["IX_TUNE_ATM_FAST"] if v["IX_TUNE_ATM_ACCUM"] else 8
            atm_block = 4 * (2 * 16 * v["IX_TUNE_ATM_FAST"] + 4 * v["IX_TUNE_ATM_FAST"] + 2 * 16 * rounds + sums)
            assert atm_block <= 48 * 1024
            assert (atm_block + 1024) * v["IX_TUNE_ATM_MIN_BLOCKS"] <= 228 * 1024
            assert 0.0 < v["IX_TUNE_PAIR_SKIN"] < 0.5 and 0.0 < v["IX_TUNE_SITE_SKIN"] < 0.5


def test_build_passes_the_tuned_values(tmp_path, monkeypatch):
    tuning = tmp_path / "tuning.json"
    tuning.write_text(json.dumps({"chosen": {"IX_TUNE_PAIR_ROUND": 64, "IX_TUNE_PAIR_SKIN": 0.08}}))
    monkeypatch.setattr(build_lib, "TUNING", tuning)
    cmd = build_lib.compile_command(tmp_path / "lib.so")
    assert "-DIX_TUNE_PAIR_ROUND=64" in cmd and "-DIX_TUNE_PAIR_SKIN=0.08f" in cmd
    assert "arch=compute_100a,code=sm_100a" in " ".join(cmd)
    explicit = build_lib.compile_command(tmp_path / "lib.so", {"IX_TUNE_PAIR_ILP": 1})
    assert "-DIX_TUNE_PAIR_ILP=1" in explicit and not any("PAIR_ROUND" in a for a in explicit)


def test_selection_keeps_the_current_values_within_the_margin(tmp_path):
    cur = dict(tune.DEFAULTS)
    other = dict(cur, IX_TUNE_PAIR_ROUND=64)
    assert tune.select([(1.0, cur), (0.995, other)], cur) == cur             # 0.5%: noise
    assert tune.select([(1.0, cur), (0.95, other)], cur) == other            # 5%: kept
    assert tune.select([(float("inf"), cur), (0.95, other)], cur) == other   # the current values failed the check
    record = {"chosen": {}, "measurements": [
        {"group": "pair tiles", "values": {"IX_TUNE_PAIR_ROUND": 128},
         "measured": {"md_step_ms": 0.30, "clusters_ms": 0.30, "oracle_energy_error": 1e-7,
                      "oracle_force_error": 1e-6}},
        {"group": "pair tiles", "values": {"IX_TUNE_PAIR_ROUND": 64},
         "measured": {"md_step_ms": 0.25, "clusters_ms": 0.30, "oracle_energy_error": 1e-7,
                      "oracle_force_error": 1e-6}},
        {"group": "pair table", "values": {"IX_TUNE_PAIR_SHARED_TABLE_BYTES": 0},
         "measured": {"md_step_ms": 0.25, "oracle_energy_error": 1e-7, "oracle_force_error": 1e-6}},
        {"group": "pair table", "values": {"IX_TUNE_PAIR_SHARED_TABLE_BYTES": 1024},
         "measured": {"md_step_ms": 0.249, "oracle_energy_error": 1e-7, "oracle_force_error": 1e-6}},
        {"group": "pair table", "values": {"IX_TUNE_PAIR_SHARED_TABLE_BYTES": 2048},
         "measured": {"md_step_ms": 0.20, "oracle_energy_error": 1e-3, "oracle_force_error": 1e-6}}]}
    path = tmp_path / "tuning.json"
    path.write_text(json.dumps(record))
    chosen = tune.reselect(path)
    assert chosen["IX_TUNE_PAIR_ROUND"] == 64 and chosen["IX_TUNE_PAIR_SHARED_TABLE_BYTES"] == 0
    assert json.loads(path.read_text())["chosen"] == chosen


def test_candidates_are_checked_against_the_shipped_build():
    base = {"md_step_ms": 0.2, "energy_error": 1e-7, "force_error": 1e-6}
    assert tune.agrees(base)
    assert not tune.agrees(dict(base, energy_error=6e-7))       # half the 1e-6 energy bar
    assert not tune.agrees(dict(base, force_error=6e-6))        # half the 1e-5 force bar
    with_clusters = dict(base, clusters_energy_error=1e-7, clusters_force_error=1e-6)
    assert tune.agrees(with_clusters)
    assert not tune.agrees(dict(with_clusters, clusters_energy_error=1e-6))
    assert tune.objective(dict(with_clusters, clusters_ms=0.3), True) == 0.2 + 0.3
    assert tune.objective(dict(base, force_error=1e-4), False) == float("inf")
    # measurements recorded against the FP64 oracle keep the full bar
    assert tune.agrees({"oracle_energy_error": 9e-7, "oracle_force_error": 9e-6})
    # the error measures: relative RMS forces, and per cluster the total energy on the scale of its terms
    import numpy as np
    ref = np.ones((4, 3))
    assert abs(tune.force_error(ref * (1 + 1e-6), ref) - 1e-6) < 1e-12
    e_ref = np.array([[10.0, -10.0, 1.0, 0.0], [5.0, 0.0, 0.0, 0.0]])
    e = e_ref.copy()
    e[0, 2] += 2.1e-6                                        # 1e-7 of the first cluster's 21 kJ/mol of terms
    assert abs(tune.batch_energy_error(e, e_ref) - 1e-7) < 1e-12
    # the tuner runs the library only: the oracle is the tests' checker
    assert "pyoracle" not in (PKG / "tune.py").read_text()
