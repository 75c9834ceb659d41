"""XML serialization of the four short-range forces and of a System, in OpenMM's XmlSerializer layout.

The element and attribute names, the version number and the defaults on reading are those of the reference's
serialization proxies (serialization/src/InteraxDispersionForceProxy.cpp:42-97, InteraxExchangeForceProxy.cpp:42-95,
InteraxShortRangeForceProxy.cpp:42-95, InteraxThreeBodyForceProxy.cpp:42-97): a force is an element with the
proxy's type name in its "type" attribute, its settings as attributes, and child elements Particles/Particle and
Exclusions/Exclusion (pair forces) or Sites/Site/Particle (three-body).  Doubles are written with 17 significant
digits, booleans as 1/0, as OpenMM's SerializationNode does, so documents round-trip exactly and files written by the
reference read here.
"""
import xml.etree.ElementTree as ET

from .forces import (OpenMMException, InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                     InteraxThreeBodyForce, System)

_VERSION = 1


def _d(x):
    return "%.17g" % float(x)


def _b(x):
    return "1" if x else "0"


def _get(node, name, default=None):
    value = node.get(name)
    if value is None:
        if default is None:
            raise OpenMMException(f"Unknown property '{name}' in node '{node.tag}'")
        return default
    return value


def _getd(node, name, default=None):
    return float(_get(node, name, None if default is None else str(default)))


def _geti(node, name, default=None):
    return int(float(_get(node, name, None if default is None else str(default))))


def _getb(node, name):
    v = _get(node, name).strip().lower()
    if v in ("1", "true"):
        return True
    if v in ("0", "false"):
        return False
    raise OpenMMException(f"Property '{name}' is not a boolean")


def _child(node, tag):
    c = node.find(tag)
    if c is None:
        raise OpenMMException(f"Unknown child '{tag}' in node '{node.tag}'")
    return c


def _pair_common(node, force):
    node.set("version", str(_VERSION))
    node.set("forceGroup", str(force.getForceGroup()))
    node.set("name", force.getName())
    node.set("method", str(int(force.getNonbondedMethod())))
    node.set("cutoff", _d(force.getCutoffDistance()))
    if not isinstance(force, InteraxDispersionForce):
        node.set("overlapMethod", str(int(force.getOverlapMethod())))
    node.set("useSwitchingFunction", _b(force.getUseSwitchingFunction()))
    node.set("switchingDistance", _d(force.getSwitchingDistance()))
    node.set("alchemicalParameter", force.getAlchemicalParameterName())
    node.set("softcoreRadius", _d(force.getSoftcoreRadius()))


def _exclusions(node, force):
    ex = ET.SubElement(node, "Exclusions")
    for i in range(force.getNumExclusions()):
        p1, p2 = force.getExclusionParticles(i)
        ET.SubElement(ex, "Exclusion", {"p1": str(p1), "p2": str(p2)})


_PARTICLE_FIELDS = {InteraxDispersionForce: ("m1", "m2", "m3", "alpha", "width"),
                    InteraxExchangeForce: ("amplitude", "width"),
                    InteraxShortRangeForce: ("k", "l", "width")}


def _serialize_force(force, tag="Force"):
    node = ET.Element(tag)
    cls = type(force)
    if isinstance(force, InteraxThreeBodyForce):
        node.set("type", "InteraxThreeBodyForce")
        node.set("version", str(_VERSION))
        node.set("forceGroup", str(force.getForceGroup()))
        node.set("name", force.getName())
        node.set("cutoff", _d(force.getCutoffDistance()))
        node.set("scaleFactor", _d(force.getScaleFactor()))
        node.set("usesPeriodic", _b(force.usesPeriodicBoundaryConditions()))
        node.set("alchemicalParameter", force.getAlchemicalParameterName())
        node.set("dampingMethod", str(int(force.getDampingMethod())))
        node.set("dampingScale", _d(force.getDampingScale()))
        node.set("centroidDampingRadius", _d(force.getCentroidDampingRadius()))
        sites = ET.SubElement(node, "Sites")
        for i in range(force.getNumSites()):
            particles, alpha, frequency, width, molecule, alch = force.getSiteParameters(i)
            site = ET.SubElement(sites, "Site", {"alpha": _d(alpha), "frequency": _d(frequency), "width": _d(width),
                                                 "molecule": str(molecule), "alchemical": _b(alch)})
            for p in particles:
                ET.SubElement(site, "Particle", {"index": str(p)})
        return node
    base = next((c for c in _PARTICLE_FIELDS if isinstance(force, c)), None)
    if base is None:
        raise OpenMMException(f"There is no serialization proxy registered for type {cls.__name__}")
    node.set("type", base.__name__)
    _pair_common(node, force)
    if base is InteraxDispersionForce:
        node.set("dampingScale", _d(force.getDampingScale()))
        node.set("useLongRangeCorrection", _b(force.getUseLongRangeCorrection()))
    particles = ET.SubElement(node, "Particles")
    for i in range(force.getNumParticles()):
        params = force.getParticleParameters(i)
        attrs = {k: _d(v) for k, v in zip(_PARTICLE_FIELDS[base], params[:-1])}
        attrs["alchemical"] = _b(params[-1])
        ET.SubElement(particles, "Particle", attrs)
    _exclusions(node, force)
    return node


def _deserialize_force(node):
    kind = node.get("type", node.tag)
    if _geti(node, "version") != _VERSION:
        raise OpenMMException("Unsupported version number")
    if kind == "InteraxThreeBodyForce":
        f = InteraxThreeBodyForce()
        f.setForceGroup(_geti(node, "forceGroup", 0))
        f.setName(_get(node, "name", f.getName()))
        f.setCutoffDistance(_getd(node, "cutoff"))
        f.setScaleFactor(_getd(node, "scaleFactor"))
        f.setUsesPeriodicBoundaryConditions(_getb(node, "usesPeriodic"))
        f.setAlchemicalParameterName(_get(node, "alchemicalParameter"))
        f.setDampingMethod(_geti(node, "dampingMethod"))
        f.setDampingScale(_getd(node, "dampingScale"))
        f.setCentroidDampingRadius(_getd(node, "centroidDampingRadius"))
        for site in _child(node, "Sites"):
            particles = [_geti(p, "index") for p in site]
            f.addSite(particles, _getd(site, "alpha"), _getd(site, "frequency"), _getd(site, "width"),
                      _geti(site, "molecule"), _getb(site, "alchemical"))
        return f
    classes = {c.__name__: c for c in _PARTICLE_FIELDS}
    if kind not in classes:
        raise OpenMMException(f"There is no serialization proxy registered for type {kind}")
    cls = classes[kind]
    f = cls()
    f.setForceGroup(_geti(node, "forceGroup", 0))
    f.setName(_get(node, "name", f.getName()))
    f.setNonbondedMethod(_geti(node, "method"))
    f.setCutoffDistance(_getd(node, "cutoff"))
    if cls is not InteraxDispersionForce:
        f.setOverlapMethod(_geti(node, "overlapMethod"))
    f.setUseSwitchingFunction(_getb(node, "useSwitchingFunction"))
    f.setSwitchingDistance(_getd(node, "switchingDistance"))
    f.setAlchemicalParameterName(_get(node, "alchemicalParameter"))
    f.setSoftcoreRadius(_getd(node, "softcoreRadius"))
    if cls is InteraxDispersionForce:
        f.setDampingScale(_getd(node, "dampingScale"))
        f.setUseLongRangeCorrection(_getb(node, "useLongRangeCorrection"))
    for p in _child(node, "Particles"):
        f.addParticle(*[_getd(p, k) for k in _PARTICLE_FIELDS[cls]], _getb(p, "alchemical"))
    for e in _child(node, "Exclusions"):
        f.addExclusion(_geti(e, "p1"), _geti(e, "p2"))
    return f


def _serialize_system(system):
    node = ET.Element("System", {"type": "System", "version": "1"})
    box = ET.SubElement(node, "PeriodicBoxVectors")
    for tag, v in zip("ABC", system.getDefaultPeriodicBoxVectors()):
        ET.SubElement(box, tag, {"x": _d(v[0]), "y": _d(v[1]), "z": _d(v[2])})
    particles = ET.SubElement(node, "Particles")
    for i in range(system.getNumParticles()):
        ET.SubElement(particles, "Particle", {"mass": _d(system.getParticleMass(i))})
    ET.SubElement(node, "Constraints")
    forces = ET.SubElement(node, "Forces")
    for force in system._forces:
        forces.append(_serialize_force(force))
    return node


def _deserialize_system(node):
    system = System()
    box = node.find("PeriodicBoxVectors")
    if box is not None:
        system.setDefaultPeriodicBoxVectors(*[(_getd(box.find(t), "x"), _getd(box.find(t), "y"),
                                               _getd(box.find(t), "z")) for t in "ABC"])
    for p in _child(node, "Particles"):
        system.addParticle(_getd(p, "mass"))
    forces = node.find("Forces")
    for f in (forces if forces is not None else []):
        kind = f.get("type")
        if kind in ("InteraxDispersionForce", "InteraxExchangeForce", "InteraxShortRangeForce", "InteraxThreeBodyForce"):
            system.addForce(_deserialize_force(f))
    return system


class XmlSerializer:
    """serialize(object) -> XML string; deserialize(string) -> object (a System or one of the four forces)."""

    @staticmethod
    def serialize(obj):
        node = _serialize_system(obj) if isinstance(obj, System) else _serialize_force(obj)
        ET.indent(node, space="\t")
        return '<?xml version="1.0" ?>\n' + ET.tostring(node, encoding="unicode") + "\n"

    @staticmethod
    def deserialize(text):
        try:
            node = ET.fromstring(text)
        except ET.ParseError as e:
            raise OpenMMException(f"Error parsing XML: {e}")
        if node.get("type") == "System" or node.tag == "System":
            return _deserialize_system(node)
        return _deserialize_force(node)

    serializeSystem = serialize
    deserializeSystem = deserialize
