"""Context and State: evaluate a System's InteraxFF short-range forces on a B200 through the C ABI.

Mirrors what the reference does inside an OpenMM Context for these forces: ForceImpl::initialize validates each
force and creates its kernel (InteraxPairForceImpl.h:73-77, InteraxThreeBodyForceImpl.cpp:42-62), getState() runs
calcForcesAndEnergy of the forces in the requested groups (InteraxPairForceImpl.h:84-88), and
updateParametersInContext() copies new parameters (InteraxPairForceImpl.h:97-100).  The context parameters default
to 1 for each alchemical parameter a force with alchemical particles defines (InteraxPairForce.cpp:138-146).
"""
import ctypes

import numpy as np

from . import _capi
from .forces import (OpenMMException, InteraxPairForce, InteraxDispersionForce, InteraxExchangeForce,
                     InteraxShortRangeForce, InteraxThreeBodyForce)


class Platform:
    """The single platform of this package: one B200 GPU, selected by its CUDA device index."""

    def __init__(self, device=0):
        self.device = int(device)

    @staticmethod
    def getName():
        return "B200"


class State:
    def __init__(self, energy, forces, term_energies, positions=None):
        self._energy = energy
        self._forces = forces
        self._terms = term_energies
        self._positions = positions

    def getPotentialEnergy(self):
        if self._energy is None:
            raise OpenMMException("Invoked getPotentialEnergy() on a State which does not contain energy.")
        return self._energy

    def getForces(self, asNumpy=True):
        if self._forces is None:
            raise OpenMMException("Invoked getForces() on a State which does not contain forces.")
        return self._forces

    def getPositions(self, asNumpy=True):
        return self._positions

    def getTermEnergies(self):
        """Energies of the dispersion, exchange, short-range and three-body terms evaluated."""
        return self._terms


def _term_index(force):
    for t, cls in enumerate((InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce)):
        if isinstance(force, cls):
            return t
    return 3 if isinstance(force, InteraxThreeBodyForce) else None


def _pair_settings(force, n):
    if force.getNumParticles() != n:
        raise OpenMMException(f"{type(force).__name__} must have exactly as many particles as the System it "
                              "belongs to.")
    ex = _capi.arr(force._exclusion_array(), np.int32)
    s = _capi.PairSettings(force.getNonbondedMethod(), force.getCutoffDistance(),
                           int(force.getUseSwitchingFunction()), force.getSwitchingDistance(),
                           force.getSoftcoreRadius(), force.getForceGroup(),
                           force.getAlchemicalParameterName().encode(), len(ex), _capi.ptr(ex))
    return s, ex


def calcLongRangeCorrection(force):
    """Long-range correction coefficients (coefficient, alchemicalCoefficient) of an InteraxDispersionForce, as
    InteraxDispersionForceImpl::calcLongRangeCorrection (openmmapi/src/InteraxDispersionForceImpl.cpp:86-149): the
    correction energy is (coefficient + lambda alchemicalCoefficient) / V.  Host-side FP64; needs no GPU."""
    lib = _capi.lib()
    n = force.getNumParticles()
    s, ex = _pair_settings(force, n)
    params = _capi.arr(force._params_array(), np.float64)
    alch = _capi.arr(force._alch_array(), np.uint8)
    coef, alch_coef = ctypes.c_double(), ctypes.c_double()
    rc = lib.ix_dispersion_long_range_correction(n, _capi.ptr(params), _capi.ptr(alch), ctypes.byref(s),
                                                 force.getDampingScale(), int(force.getUseLongRangeCorrection()),
                                                 ctypes.byref(coef), ctypes.byref(alch_coef))
    if rc != 0:
        raise OpenMMException(lib.ix_last_error(None).decode())
    return coef.value, alch_coef.value


def describe_forces(lib, handle, system, check, keep=None):
    """Describe a System's InteraxFF forces to a context or request handle with the ix_add_* functions (what the
    reference's kernels' initialize() receive, InteraxKernels.h:64-67, 99-102, 134-137, 169-172).  Returns
    {term index: force} and the alchemical parameter names that have alchemical particles or sites.  `keep`, if
    given, receives every array the calls point into (for callers that replay the calls later)."""
    n = system.getNumParticles()
    keep = [] if keep is None else keep
    forces, names = {}, []
    for force in system._forces:
        t = _term_index(force)
        if t is None:
            continue
        if t < 3:
            s, ex = _pair_settings(force, n)
            params = _capi.arr(force._params_array(), np.float64)
            alch = _capi.arr(force._alch_array(), np.uint8)
            keep += [s, ex, params, alch]
            if t == 0:
                rc = lib.ix_add_dispersion(handle, ctypes.byref(s), _capi.ptr(params), _capi.ptr(alch),
                                           force.getDampingScale(), int(force.getUseLongRangeCorrection()))
            elif t == 1:
                rc = lib.ix_add_exchange(handle, ctypes.byref(s), _capi.ptr(params), _capi.ptr(alch),
                                         force.getOverlapMethod())
            else:
                rc = lib.ix_add_short_range(handle, ctypes.byref(s), _capi.ptr(params), _capi.ptr(alch),
                                            force.getOverlapMethod())
        else:
            off, part, params, mol, alch = force._site_arrays()
            arrays = [_capi.arr(off, np.int32), _capi.arr(part, np.int32), _capi.arr(params, np.float64),
                      _capi.arr(mol, np.int32), _capi.arr(alch, np.uint8)]
            keep += arrays
            rc = lib.ix_add_three_body(
                handle, force.getNumSites(), *[_capi.ptr(a) for a in arrays], force.getCutoffDistance(),
                force.getScaleFactor(), force.getDampingMethod(), force.getDampingScale(),
                force.getCentroidDampingRadius(),
                int(force.usesPeriodicBoundaryConditions()), force.getAlchemicalParameterName().encode(),
                force.getForceGroup())
        check(rc)
        if alch.any():
            names.append(force.getAlchemicalParameterName())
        forces[t] = force
    return forces, names


class Context:
    # relative tolerance of the MD loop's constraints (squared distances, stretching rate per ps)
    constraintTolerance = 1e-10

    def __init__(self, system, integrator=None, platform=None, properties=None):
        self._system = system
        self._platform = platform if isinstance(platform, Platform) else Platform(
            (properties or {}).get("DeviceIndex", 0))
        self._lib = _capi.lib()
        self._ctx = ctypes.c_void_p()
        self._positions = None
        self._box = np.array(system.getDefaultPeriodicBoxVectors(), dtype=np.float64)
        self._parameters = {}
        self._forces = {}
        self._create()

    # -- setup ------------------------------------------------------------------------------------------------
    def _check(self, rc):
        if rc != _capi.IX_OK:
            msg = self._lib.ix_last_error(self._ctx if self._ctx else None).decode()
            raise OpenMMException(msg)

    def _create(self):
        system = self._system
        n = system.getNumParticles()
        box = _capi.arr(self._box.reshape(9), np.float64)
        rc = self._lib.ix_ctx_create(n, self._platform.device, _capi.ptr(box), ctypes.byref(self._ctx))
        if rc != _capi.IX_OK:
            msg = self._lib.ix_last_error(None).decode()
            self._ctx = ctypes.c_void_p()
            raise OpenMMException(msg)
        self._forces, names = describe_forces(self._lib, self._ctx, system, self._check)
        for name in names:
            self._parameters.setdefault(name, 1.0)
        if system.getNumConstraints():
            cons = [system.getConstraintParameters(i) for i in range(system.getNumConstraints())]
            pairs = _capi.arr([(a, b) for a, b, _ in cons], np.int32)
            dist = _capi.arr([d for _, _, d in cons], np.float64)
            self._check(self._lib.ix_md_set_constraints(self._ctx, len(cons), _capi.ptr(pairs), _capi.ptr(dist),
                                                        self.constraintTolerance))

    def __del__(self):
        if getattr(self, "_ctx", None) and self._ctx.value:
            self._lib.ix_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    # -- state ------------------------------------------------------------------------------------------------
    def getSystem(self):
        return self._system

    def getPlatform(self):
        return self._platform

    def setPositions(self, positions):
        pos = _capi.arr(np.asarray(positions, dtype=np.float64).reshape(-1, 3), np.float64)
        if len(pos) != self._system.getNumParticles():
            raise OpenMMException("Called setPositions() on a Context with the wrong number of positions")
        self._positions = pos.copy()
        self._check(self._lib.ix_set_positions(self._ctx, _capi.ptr(pos), _capi.ptr(self._box_array())))

    def _box_array(self):
        return _capi.arr(self._box.reshape(9), np.float64)

    def setPeriodicBoxVectors(self, a, b, c):
        self._box = np.array([a, b, c], dtype=np.float64)
        if self._positions is not None:
            self._check(self._lib.ix_set_positions(self._ctx, _capi.ptr(self._positions), _capi.ptr(self._box_array())))

    def getPeriodicBoxVectors(self):
        return self._box.copy()

    def setParameter(self, name, value):
        if name not in self._parameters:
            raise OpenMMException("Called setParameter() with invalid parameter name")
        self._parameters[name] = float(value)
        self._check(self._lib.ix_set_parameter(self._ctx, name.encode(), float(value)))

    def getParameter(self, name):
        if name not in self._parameters:
            raise OpenMMException("Called getParameter() with invalid parameter name")
        return self._parameters[name]

    def getParameters(self):
        return dict(self._parameters)

    def getState(self, getEnergy=True, getForces=True, groups=0xFFFFFFFF, getPositions=False):
        if self._positions is None:
            raise OpenMMException("Particle positions have not been set")
        n = self._system.getNumParticles()
        terms = np.zeros(4)
        energy = ctypes.c_double()
        forces = np.zeros((n, 3)) if getForces else None
        groups = int(groups) & 0xFFFFFFFF
        if groups >= 1 << 31:
            groups -= 1 << 32
        self._check(self._lib.ix_compute(self._ctx, groups, int(getForces), int(getEnergy), _capi.ptr(terms),
                                         ctypes.byref(energy), _capi.ptr(forces)))
        return State(energy.value if getEnergy else None, forces, terms,
                     self._positions.copy() if getPositions else None)

    def setListCapacity(self, pairTiles=0, siteNeighbors=0):
        """Capacities of the pair list (tiles) and of the three-body lists (entries per site) at their next
        allocation; 0 = estimated from the density.  The lists grow when they overflow, and a small capacity forces
        that path (ix_set_list_capacity)."""
        self._check(self._lib.ix_set_list_capacity(self._ctx, int(pairTiles), int(siteNeighbors)))

    def getListStats(self):
        """(pair-list tiles, three-body entries per site, MD steps reruns after an overflow) (ix_get_list_stats)."""
        a, b, c = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_longlong()
        self._check(self._lib.ix_get_list_stats(self._ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def getCounts(self):
        """Interacting pairs and triples of the last evaluation."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self._lib.ix_get_counts(self._ctx, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def reinitialize(self, preserveState=False):
        positions, params = self._positions, dict(self._parameters)
        if self._ctx.value:
            self._lib.ix_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()
        self._parameters = {}
        self._forces = {}
        self._create()
        if preserveState:
            for k, v in params.items():
                if k in self._parameters:
                    self.setParameter(k, v)
            if positions is not None:
                self.setPositions(positions)

    def _update_force(self, force):
        t = _term_index(force)
        if t is None or self._forces.get(t) is not force:
            raise OpenMMException("updateParametersInContext: the force is not part of this Context")
        L = self._lib
        if t < 3:
            if force.getNumParticles() != self._system.getNumParticles():
                raise OpenMMException("updateParametersInContext: The number of particles has changed")
            params = _capi.arr(force._params_array(), np.float64)
            if t == 0:
                self._check(L.ix_update_dispersion(self._ctx, _capi.ptr(params), force.getDampingScale()))
            elif t == 1:
                self._check(L.ix_update_exchange(self._ctx, _capi.ptr(params), force.getOverlapMethod()))
            else:
                self._check(L.ix_update_short_range(self._ctx, _capi.ptr(params), force.getOverlapMethod()))
        else:
            off, part, params, mol, alch = force._site_arrays()
            self._check(L.ix_update_three_body(self._ctx, _capi.ptr(_capi.arr(params, np.float64)),
                                               force.getScaleFactor(), force.getDampingScale(),
                                               force.getCentroidDampingRadius()))

    def computeWindows(self, name, values, getForces=True):
        """Term energies (num_windows x 4) and, optionally, forces (num_windows x n x 3) of the current positions at
        each value of the alchemical parameter `name` (the C ABI's ix_compute_windows).  The parameter keeps its
        value."""
        values = _capi.arr(np.asarray(values, dtype=np.float64).reshape(-1), np.float64)
        n = self._system.getNumParticles()
        energies = np.zeros((len(values), 4))
        forces = np.zeros((len(values), n, 3)) if getForces else None
        self._check(self._lib.ix_compute_windows(self._ctx, name.encode(), len(values), _capi.ptr(values),
                                                 _capi.ptr(energies), _capi.ptr(forces) if getForces else None))
        return (energies, forces) if getForces else energies

    # -- MD -----------------------------------------------------------------------------------------------------
    def runVelocityVerlet(self, steps, dt, velocities):
        """Run `steps` velocity-Verlet steps of `dt` ps on the device; returns (positions, velocities, energy)."""
        n = self._system.getNumParticles()
        masses = _capi.arr([self._system.getParticleMass(i) for i in range(n)], np.float64)
        self._check(self._lib.ix_md_set_masses(self._ctx, _capi.ptr(masses)))
        pos = self._positions.copy()
        vel = _capi.arr(velocities, np.float64).copy()
        e = ctypes.c_double()
        self._check(self._lib.ix_md_run(self._ctx, int(steps), float(dt), _capi.ptr(pos), _capi.ptr(vel),
                                        ctypes.byref(e)))
        self._positions = pos
        return pos, vel, e.value
