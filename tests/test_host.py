"""Host-side tests that need no GPU: the C ABI library loads and exports every declared symbol, the Force classes
validate as the reference's do, and a context refuses to run without a Blackwell GPU (no CPU fallback)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "interax_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ix_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from interaxplugin import _capi
    lib = ctypes.CDLL(str(_capi.LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name


def test_version_string():
    from interaxplugin import _capi
    assert b"sm_100a" in _capi.lib().ix_version()


def test_context_needs_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from interaxplugin import Context, OpenMMException
    from interaxplugin import workloads as W
    system, pos, box = W.water_box(8, 1.0, 0.45, seed=0, three_body=False)
    with pytest.raises(OpenMMException, match="device"):
        Context(system)


def test_force_api_defaults_and_validation():
    from interaxplugin import (InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                               InteraxThreeBodyForce, OpenMMException)
    d = InteraxDispersionForce()
    assert d.getNonbondedMethod() == 0 and d.getCutoffDistance() == 1.0 and d.getSwitchingDistance() == -1.0
    assert d.getAlchemicalParameterName() == "lambda_sterics" and d.getDampingScale() == 1.0
    assert not d.getUseLongRangeCorrection()
    with pytest.raises(OpenMMException, match="soft-core radius cannot be negative"):
        d.setSoftcoreRadius(-0.1)
    with pytest.raises(OpenMMException, match="nonbonded method"):
        d.setNonbondedMethod(3)
    x = InteraxExchangeForce()
    assert x.getOverlapMethod() == InteraxExchangeForce.Exact
    with pytest.raises(OpenMMException, match="overlap method"):
        x.setOverlapMethod(1)
    s = InteraxShortRangeForce()
    s.addParticle(1.0, 2.0, 0.02, True)
    assert s.getParticleParameters(0) == (1.0, 2.0, 0.02, True)
    with pytest.raises(OpenMMException):
        s.getParticleParameters(1)
    t = InteraxThreeBodyForce()
    assert t.getCutoffDistance() == 1.2 and t.getScaleFactor() == 1.0 and t.getDampingMethod() == 0
    assert not t.usesPeriodicBoundaryConditions()
    with pytest.raises(OpenMMException, match="centroid damping radius"):
        t.setCentroidDampingRadius(-1)
    with pytest.raises(OpenMMException, match="damping method"):
        t.setDampingMethod(2)
    t.addSite([0, 1], 0.004, 900.0)
    assert t.getSiteParameters(0) == ([0, 1], 0.004, 900.0, 0.0, -1, False)


def test_workloads_shapes():
    from interaxplugin import workloads as W
    system, pos, box = W.water_box(216, 1.865, 0.9, seed=1, three_body_cutoff=0.6)
    assert pos.shape == (648, 3) and system.getNumParticles() == 648
    assert system.getForce(0).getNumExclusions() == 3 * 216
    oh = np.linalg.norm(pos[1] - pos[0])
    assert oh == pytest.approx(0.09572)
    system, pos, _ = W.water_cluster(10, seed=2)
    assert pos.shape == (30, 3) and system.getForce(0).getNonbondedMethod() == 0
