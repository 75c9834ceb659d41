"""XML serialization of the four forces and of a System (interaxplugin.XmlSerializer), following the reference's own
serialization tests (serialization/tests/TestSerializeInterax{Dispersion,Exchange,ShortRange,ThreeBody}Force.cpp):
every setting and parameter survives a round trip exactly, serializing the copy gives the same XML, defaults are kept,
and an unsupported version number is rejected."""
import numpy as np
import pytest

import pyoracle
from interaxplugin import (InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                           InteraxThreeBodyForce, OpenMMException, XmlSerializer)
from interaxplugin import workloads as W


def _pair_settings(force):
    force.setForceGroup(3)
    force.setName("custom name")
    force.setNonbondedMethod(1)
    force.setCutoffDistance(1.1)
    force.setUseSwitchingFunction(True)
    force.setSwitchingDistance(0.95)
    force.setAlchemicalParameterName("lambda_test")
    force.setSoftcoreRadius(0.12)
    force.addExclusion(0, 1)
    force.addExclusion(2, 1)


def _dispersion():
    f = InteraxDispersionForce()
    _pair_settings(f)
    f.setDampingScale(1.37)
    f.setUseLongRangeCorrection(True)
    f.addParticle(0.0012345678901234567, 1.5e-5, 2.2e-7, 0.8, 0.031)
    f.addParticle(0.002, 3e-5, 4e-7, 0.0, 0.02, True)
    f.addParticle(0.0, 0.0, 0.0, 0.0, 0.0, False)
    return f


def _exchange(method=2):
    f = InteraxExchangeForce()
    _pair_settings(f)
    f.setOverlapMethod(method)
    f.addParticle(10.326424719450545, 0.0248302193400194)
    f.addParticle(1.0254403205662432, 0.019763296864870033, True)
    f.addParticle(0.0, 0.0, False)
    return f


def _short_range(method=0):
    f = InteraxShortRangeForce()
    _pair_settings(f)
    f.setOverlapMethod(method)
    f.addParticle(3.3, -0.7, 0.025)
    f.addParticle(1.1, -0.2, 0.03, True)
    f.addParticle(0.0, 0.0, 0.0)
    return f


def _three_body():
    f = InteraxThreeBodyForce()
    f.setForceGroup(5)
    f.setName("atm")
    f.setCutoffDistance(0.77)
    f.setScaleFactor(1.25)
    f.setUsesPeriodicBoundaryConditions(True)
    f.setAlchemicalParameterName("lambda_atm")
    f.setDampingMethod(1)
    f.setDampingScale(1.1)
    f.setCentroidDampingRadius(0.3)
    f.addSite([0, 1, 2], 0.004087456746801944, 911.0681141195369, 0.03, 7, True)
    f.addSite([3], 0.0016246535729804365, 1262.664320774599, 0.025)
    return f


def _state(f):
    if isinstance(f, InteraxThreeBodyForce):
        return (f.getForceGroup(), f.getName(), f.getCutoffDistance(), f.getScaleFactor(),
                f.usesPeriodicBoundaryConditions(), f.getAlchemicalParameterName(), f.getDampingMethod(),
                f.getDampingScale(), f.getCentroidDampingRadius(),
                [f.getSiteParameters(i) for i in range(f.getNumSites())])
    extra = (f.getDampingScale(), f.getUseLongRangeCorrection()) if isinstance(f, InteraxDispersionForce) \
        else (f.getOverlapMethod(),)
    return (type(f), f.getForceGroup(), f.getName(), f.getNonbondedMethod(), f.getCutoffDistance(),
            f.getUseSwitchingFunction(), f.getSwitchingDistance(), f.getAlchemicalParameterName(),
            f.getSoftcoreRadius(), extra, [f.getParticleParameters(i) for i in range(f.getNumParticles())],
            [f.getExclusionParticles(i) for i in range(f.getNumExclusions())])


@pytest.mark.parametrize("make", [_dispersion, lambda: _exchange(0), lambda: _exchange(2), lambda: _short_range(0),
                                  lambda: _short_range(2), _three_body])
def test_round_trip(make):
    force = make()
    xml = XmlSerializer.serialize(force)
    copy = XmlSerializer.deserialize(xml)
    assert type(copy) is type(force)
    assert _state(copy) == _state(force)
    assert XmlSerializer.serialize(copy) == xml


@pytest.mark.parametrize("cls", [InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                                 InteraxThreeBodyForce])
def test_defaults(cls):
    force = cls()
    copy = XmlSerializer.deserialize(XmlSerializer.serialize(force))
    assert _state(copy) == _state(force)
    assert copy.getAlchemicalParameterName() == "lambda_sterics"


@pytest.mark.parametrize("cls", [InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                                 InteraxThreeBodyForce])
def test_unsupported_version(cls):
    xml = XmlSerializer.serialize(cls())
    assert 'version="1"' in xml
    with pytest.raises(OpenMMException, match="Unsupported version number"):
        XmlSerializer.deserialize(xml.replace('version="1"', 'version="2"', 1))


def test_document_in_the_proxy_layout():
    """A document written in the reference proxy's layout (attributes of InteraxExchangeForceProxy::serialize)."""
    xml = ('<?xml version="1.0" ?>\n<Force alchemicalParameter="lambda_x" cutoff="0.9" forceGroup="2" method="1" '
           'name="ex" overlapMethod="2" softcoreRadius="0.1" switchingDistance="-1" type="InteraxExchangeForce" '
           'useSwitchingFunction="0" version="1">\n\t<Particles>\n\t\t<Particle alchemical="1" amplitude="12.5" '
           'width="22.25"/>\n\t\t<Particle alchemical="0" amplitude="3" width="31"/>\n\t</Particles>\n\t<Exclusions>'
           '\n\t\t<Exclusion p1="0" p2="1"/>\n\t</Exclusions>\n</Force>\n')
    f = XmlSerializer.deserialize(xml)
    assert isinstance(f, InteraxExchangeForce)
    assert (f.getForceGroup(), f.getName(), f.getNonbondedMethod(), f.getOverlapMethod()) == (2, "ex", 1, 2)
    assert f.getParticleParameters(0) == (12.5, 22.25, True)
    assert f.getExclusionParticles(0) == (0, 1)


def test_system_round_trip_evaluates_the_same():
    system, pos, box = W.water_box(24, 1.0, 0.45, seed=3, three_body_cutoff=0.4, alchemical_waters=[1, 2],
                                   softcore_radius=0.1)
    copy = XmlSerializer.deserialize(XmlSerializer.serialize(system))
    assert copy.getNumParticles() == system.getNumParticles() and copy.getNumForces() == system.getNumForces()
    assert np.array_equal(np.array(copy.getDefaultPeriodicBoxVectors()), np.array(system.getDefaultPeriodicBoxVectors()))
    assert [copy.getParticleMass(i) for i in range(copy.getNumParticles())] == \
        [system.getParticleMass(i) for i in range(system.getNumParticles())]
    e1, f1 = pyoracle.evaluate(system, pos, box, {"lambda_sterics": 0.4})
    e2, f2 = pyoracle.evaluate(copy, pos, box, {"lambda_sterics": 0.4})
    assert e1 == e2 and np.array_equal(f1, f2)
