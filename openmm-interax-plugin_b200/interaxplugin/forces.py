"""The InteraxFF short-range Force classes, with the names, defaults, arguments and errors of the plugin's C++ API.

Mirrors openmmapi/include/InteraxPairForce.h:70-239, InteraxDispersionForce.h:70-182, InteraxExchangeForce.h:60-160,
InteraxShortRangeForce.h:59-162 and InteraxThreeBodyForce.h:75-258 (and the SWIG module python/interaxplugin.i,
which exposes the same class and method names).  These objects only hold parameters; a Context uploads them to the
device through the C-ABI, which performs the validation the reference performs at Context creation.
"""

class OpenMMException(Exception):
    """Raised where the reference throws OpenMM::OpenMMException, with the same messages."""


def _check_index(index, items):
    # ASSERT_VALID_INDEX of the reference accessors
    if index < 0 or index >= len(items):
        raise OpenMMException("Index out of range")


class Force:
    """The parts of OpenMM::Force the forces use: force group and name."""

    def __init__(self):
        self._group = 0
        self._name = type(self).__name__

    def getForceGroup(self):
        return self._group

    def setForceGroup(self, group):
        if group < 0 or group > 31:
            raise OpenMMException("Force group must be between 0 and 31")
        self._group = group

    def getName(self):
        return self._name

    def setName(self, name):
        self._name = name

    def updateParametersInContext(self, context):
        context._update_force(self)


class InteraxPairForce(Force):
    """Settings shared by the pair forces (InteraxPairForce.h:70-239, InteraxPairForce.cpp:41-111)."""
    NoCutoff = 0
    CutoffNonPeriodic = 1
    CutoffPeriodic = 2

    def __init__(self):
        super().__init__()
        self._method = self.NoCutoff
        self._cutoff = 1.0
        self._switching_distance = -1.0
        self._softcore_radius = 0.0
        self._use_switch = False
        self._alch_name = "lambda_sterics"
        self._exclusions = []
        self._particles = []

    def getNumParticles(self):
        return len(self._particles)

    def getParticleIsAlchemical(self, index):
        _check_index(index, self._particles)
        return self._particles[index][-1]

    def getNonbondedMethod(self):
        return self._method

    def setNonbondedMethod(self, method):
        if method < 0 or method > 2:
            raise OpenMMException("InteraxPairForce: Illegal value for nonbonded method")
        self._method = int(method)

    def getCutoffDistance(self):
        return self._cutoff

    def setCutoffDistance(self, distance):
        self._cutoff = float(distance)

    def getUseSwitchingFunction(self):
        return self._use_switch

    def setUseSwitchingFunction(self, use):
        self._use_switch = bool(use)

    def getSwitchingDistance(self):
        return self._switching_distance

    def setSwitchingDistance(self, distance):
        self._switching_distance = float(distance)

    def getNumExclusions(self):
        return len(self._exclusions)

    def addExclusion(self, particle1, particle2):
        self._exclusions.append((int(particle1), int(particle2)))
        return len(self._exclusions) - 1

    def getExclusionParticles(self, index):
        _check_index(index, self._exclusions)
        return self._exclusions[index]

    def setExclusionParticles(self, index, particle1, particle2):
        _check_index(index, self._exclusions)
        self._exclusions[index] = (int(particle1), int(particle2))

    def getAlchemicalParameterName(self):
        return self._alch_name

    def setAlchemicalParameterName(self, name):
        self._alch_name = str(name)

    def getSoftcoreRadius(self):
        return self._softcore_radius

    def setSoftcoreRadius(self, radius):
        if radius < 0:
            raise OpenMMException("InteraxPairForce: The soft-core radius cannot be negative")
        self._softcore_radius = float(radius)

    def usesPeriodicBoundaryConditions(self):
        return self._method == self.CutoffPeriodic

    # host-side helpers used by the Context and the oracle bridge
    def _params_array(self):
        import numpy as np
        return np.array([p[:-1] for p in self._particles], dtype=np.float64).reshape(len(self._particles), -1)

    def _alch_array(self):
        import numpy as np
        return np.array([1 if p[-1] else 0 for p in self._particles], dtype=np.uint8)

    def _exclusion_array(self):
        import numpy as np
        return np.array(self._exclusions, dtype=np.int32).reshape(-1, 2)


class InteraxDispersionForce(InteraxPairForce):
    """Tang-Toennies damped C6/C8/C10 dispersion (InteraxDispersionForce.h:70-182)."""

    def __init__(self):
        super().__init__()
        self._damping_scale = 1.0
        self._use_lrc = False

    def addParticle(self, m1, m2, m3, alpha, width, isAlchemical=False):
        self._particles.append((float(m1), float(m2), float(m3), float(alpha), float(width), bool(isAlchemical)))
        return len(self._particles) - 1

    def getParticleParameters(self, index):
        _check_index(index, self._particles)
        return self._particles[index]

    def setParticleParameters(self, index, m1, m2, m3, alpha, width, isAlchemical):
        _check_index(index, self._particles)
        self._particles[index] = (float(m1), float(m2), float(m3), float(alpha), float(width), bool(isAlchemical))

    def getDampingScale(self):
        return self._damping_scale

    def setDampingScale(self, scale):
        self._damping_scale = float(scale)

    def getUseLongRangeCorrection(self):
        return self._use_lrc

    def setUseLongRangeCorrection(self, use):
        self._use_lrc = bool(use)


class _OverlapForce(InteraxPairForce):
    Exact = 0
    InteraxOrder2 = 2

    def __init__(self):
        super().__init__()
        self._overlap_method = self.Exact

    def getOverlapMethod(self):
        return self._overlap_method

    def setOverlapMethod(self, method):
        if method not in (self.Exact, self.InteraxOrder2):
            raise OpenMMException(f"{type(self).__name__}: Illegal value for overlap method")
        self._overlap_method = int(method)


class InteraxExchangeForce(_OverlapForce):
    """Exchange repulsion A_i A_j S(r; s_i, s_j) (InteraxExchangeForce.h:60-160)."""

    def addParticle(self, amplitude, width, isAlchemical=False):
        self._particles.append((float(amplitude), float(width), bool(isAlchemical)))
        return len(self._particles) - 1

    def getParticleParameters(self, index):
        _check_index(index, self._particles)
        return self._particles[index]

    def setParticleParameters(self, index, amplitude, width, isAlchemical):
        _check_index(index, self._particles)
        self._particles[index] = (float(amplitude), float(width), bool(isAlchemical))


class InteraxShortRangeForce(_OverlapForce):
    """Short-range correction (K_i+K_j)/2 St + (L_i+L_j)/2 St^2 (InteraxShortRangeForce.h:59-162)."""

    def addParticle(self, k, l, width, isAlchemical=False):
        self._particles.append((float(k), float(l), float(width), bool(isAlchemical)))
        return len(self._particles) - 1

    def getParticleParameters(self, index):
        _check_index(index, self._particles)
        return self._particles[index]

    def setParticleParameters(self, index, k, l, width, isAlchemical):
        _check_index(index, self._particles)
        self._particles[index] = (float(k), float(l), float(width), bool(isAlchemical))


class InteraxThreeBodyForce(Force):
    """Axilrod-Teller-Muto three-body dispersion between centroid sites (InteraxThreeBodyForce.h:75-258,
    InteraxThreeBodyForce.cpp:39-132)."""
    NoDamping = 0
    TangToennies = 1

    def __init__(self):
        super().__init__()
        self._cutoff = 1.2
        self._scale = 1.0
        self._damping_scale = 1.0
        self._centroid_radius = 0.0
        self._damping_method = self.NoDamping
        self._periodic = False
        self._alch_name = "lambda_sterics"
        self._sites = []

    def getNumSites(self):
        return len(self._sites)

    def addSite(self, particles, alpha, frequency, width=0.0, molecule=-1, isAlchemical=False):
        self._sites.append((list(int(p) for p in particles), float(alpha), float(frequency), float(width),
                            int(molecule), bool(isAlchemical)))
        return len(self._sites) - 1

    def getSiteParameters(self, index):
        _check_index(index, self._sites)
        s = self._sites[index]
        return (list(s[0]),) + s[1:]

    def setSiteParameters(self, index, particles, alpha, frequency, width, molecule, isAlchemical):
        _check_index(index, self._sites)
        self._sites[index] = (list(int(p) for p in particles), float(alpha), float(frequency), float(width),
                              int(molecule), bool(isAlchemical))

    def getCutoffDistance(self):
        return self._cutoff

    def setCutoffDistance(self, distance):
        self._cutoff = float(distance)

    def getScaleFactor(self):
        return self._scale

    def setScaleFactor(self, scale):
        self._scale = float(scale)

    def getDampingMethod(self):
        return self._damping_method

    def setDampingMethod(self, method):
        if method not in (self.NoDamping, self.TangToennies):
            raise OpenMMException("InteraxThreeBodyForce: Illegal value for damping method")
        self._damping_method = int(method)

    def getDampingScale(self):
        return self._damping_scale

    def setDampingScale(self, scale):
        self._damping_scale = float(scale)

    def getCentroidDampingRadius(self):
        return self._centroid_radius

    def setCentroidDampingRadius(self, radius):
        if radius < 0:
            raise OpenMMException("InteraxThreeBodyForce: The centroid damping radius cannot be negative")
        self._centroid_radius = float(radius)

    def setUsesPeriodicBoundaryConditions(self, periodic):
        self._periodic = bool(periodic)

    def usesPeriodicBoundaryConditions(self):
        return self._periodic

    def getAlchemicalParameterName(self):
        return self._alch_name

    def setAlchemicalParameterName(self, name):
        self._alch_name = str(name)

    # host-side helpers
    def _site_arrays(self):
        import numpy as np
        offsets = [0]
        particles = []
        for s in self._sites:
            particles += s[0]
            offsets.append(len(particles))
        params = np.array([[s[1], s[2], s[3]] for s in self._sites], dtype=np.float64).reshape(-1, 3)
        molecule = np.array([s[4] for s in self._sites], dtype=np.int32)
        alch = np.array([1 if s[5] else 0 for s in self._sites], dtype=np.uint8)
        return (np.array(offsets, dtype=np.int32), np.array(particles, dtype=np.int32), params, molecule, alch)


class System:
    """The parts of OpenMM::System the forces need: particles (masses), forces and the default box."""

    def __init__(self):
        self._masses = []
        self._forces = []
        self._constraints = []
        self._box = [(2.0, 0.0, 0.0), (0.0, 2.0, 0.0), (0.0, 0.0, 2.0)]

    def addConstraint(self, particle1, particle2, distance):
        """A distance constraint, as OpenMM's System::addConstraint; applied by the MD loop of a Context."""
        self._constraints.append((int(particle1), int(particle2), float(distance)))
        return len(self._constraints) - 1

    def getNumConstraints(self):
        return len(self._constraints)

    def getConstraintParameters(self, index):
        return self._constraints[index]

    def addParticle(self, mass):
        self._masses.append(float(mass))
        return len(self._masses) - 1

    def getNumParticles(self):
        return len(self._masses)

    def getParticleMass(self, index):
        return self._masses[index]

    def addForce(self, force):
        self._forces.append(force)
        return len(self._forces) - 1

    def getNumForces(self):
        return len(self._forces)

    def getForce(self, index):
        return self._forces[index]

    def removeForce(self, index):
        del self._forces[index]

    def setDefaultPeriodicBoxVectors(self, a, b, c):
        self._box = [tuple(map(float, a)), tuple(map(float, b)), tuple(map(float, c))]

    def getDefaultPeriodicBoxVectors(self):
        return [tuple(v) for v in self._box]

    def usesPeriodicBoundaryConditions(self):
        return any(f.usesPeriodicBoundaryConditions() for f in self._forces)


def computeC9(alpha1, frequency1, alpha2, frequency2, alpha3, frequency3):
    """C9 of a triple (openmmapi/include/internal/InteraxThreeBodyForceImpl.h:69-72)."""
    return (1.5 * alpha1 * alpha2 * alpha3 * frequency1 * frequency2 * frequency3 * (frequency1 + frequency2 + frequency3)
            / ((frequency1 + frequency2) * (frequency2 + frequency3) * (frequency3 + frequency1)))


__all__ = ["OpenMMException", "Force", "InteraxPairForce", "InteraxDispersionForce", "InteraxExchangeForce",
           "InteraxShortRangeForce", "InteraxThreeBodyForce", "System", "computeC9"]
