"""Batched evaluation of many independent non-periodic Systems on one GPU (the C ABI's ix_batch_* functions).

Every System must carry the same forces with the same settings (methods, cutoffs, switching, soft core, overlap
method, damping, alchemical parameter); particle parameters, exclusions and three-body sites may differ.  All
Systems are evaluated together by one CUDA graph; each System's energies and forces are the same as a Context of that
System alone gives.
"""
import ctypes

import numpy as np

from . import _capi
from .context import _term_index
from .forces import OpenMMException


class BatchContext:
    def __init__(self, systems, device=0):
        self._lib = _capi.lib()
        self._batch = ctypes.c_void_p()
        self._systems = list(systems)
        self._keep = []
        rc = self._lib.ix_batch_create(int(device), ctypes.byref(self._batch))
        if rc != _capi.IX_OK:
            self._batch = ctypes.c_void_p()
            raise OpenMMException(self._lib.ix_batch_last_error(None).decode())
        self._sizes = []
        for system in self._systems:
            self._add(system)
        self._offsets = np.concatenate([[0], np.cumsum(self._sizes)]).astype(np.int64)
        self._energies = np.zeros((len(self._systems), 4))
        self._forces = np.zeros((int(self._offsets[-1]), 3))

    def _check(self, rc):
        if rc != _capi.IX_OK:
            raise OpenMMException(self._lib.ix_batch_last_error(self._batch).decode())

    def _add(self, system):
        L, b = self._lib, self._batch
        n = system.getNumParticles()
        index = ctypes.c_int()
        self._check(L.ix_batch_add_system(b, n, ctypes.byref(index)))
        s = index.value
        self._sizes.append(n)
        for force in system._forces:
            t = _term_index(force)
            if t is None:
                continue
            if t < 3:
                if force.getNumParticles() != n:
                    raise OpenMMException(f"{type(force).__name__} must have exactly as many particles as the System "
                                          "it belongs to.")
                ex = _capi.arr(force._exclusion_array(), np.int32)
                st = _capi.PairSettings(force.getNonbondedMethod(), force.getCutoffDistance(),
                                        int(force.getUseSwitchingFunction()), force.getSwitchingDistance(),
                                        force.getSoftcoreRadius(), force.getForceGroup(),
                                        force.getAlchemicalParameterName().encode(), len(ex), _capi.ptr(ex))
                params = _capi.arr(force._params_array(), np.float64)
                alch = _capi.arr(force._alch_array(), np.uint8)
                if t == 0:
                    rc = L.ix_batch_add_dispersion(b, s, ctypes.byref(st), _capi.ptr(params), _capi.ptr(alch),
                                                   force.getDampingScale(), int(force.getUseLongRangeCorrection()))
                elif t == 1:
                    rc = L.ix_batch_add_exchange(b, s, ctypes.byref(st), _capi.ptr(params), _capi.ptr(alch),
                                                 force.getOverlapMethod())
                else:
                    rc = L.ix_batch_add_short_range(b, s, ctypes.byref(st), _capi.ptr(params), _capi.ptr(alch),
                                                    force.getOverlapMethod())
                self._check(rc)
            else:
                off, part, params, mol, alch = force._site_arrays()
                arrays = [_capi.arr(off, np.int32), _capi.arr(part, np.int32), _capi.arr(params, np.float64),
                          _capi.arr(mol, np.int32), _capi.arr(alch, np.uint8)]
                rc = L.ix_batch_add_three_body(
                    b, s, force.getNumSites(), *[_capi.ptr(a) for a in arrays], force.getCutoffDistance(),
                    force.getScaleFactor(), force.getDampingMethod(), force.getDampingScale(),
                    force.getCentroidDampingRadius(), int(force.usesPeriodicBoundaryConditions()),
                    force.getAlchemicalParameterName().encode(), force.getForceGroup())
                self._check(rc)

    def setParameter(self, name, value):
        self._check(self._lib.ix_batch_set_parameter(self._batch, name.encode(), float(value)))

    def compute(self, positions):
        """positions: one (n_s, 3) array per System, or the concatenation.  Returns (energies, forces): energies
        (num_systems, 4) per term in kJ/mol, forces a list of (n_s, 3) arrays in kJ/mol/nm."""
        if isinstance(positions, (list, tuple)):
            positions = np.concatenate([np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in positions])
        pos = _capi.arr(np.asarray(positions, dtype=np.float64).reshape(-1, 3), np.float64)
        if pos.shape[0] != self._offsets[-1]:
            raise OpenMMException("positions must hold every particle of every System of the batch")
        self._check(self._lib.ix_batch_compute(self._batch, _capi.ptr(pos), _capi.ptr(self._forces),
                                               _capi.ptr(self._energies)))
        forces = [self._forces[self._offsets[s]:self._offsets[s + 1]].copy() for s in range(len(self._systems))]
        return self._energies.copy(), forces

    def runVelocityVerlet(self, steps, dt, positions, velocities=None):
        """steps[s] velocity-Verlet steps of dt ps for System s, all Systems at once on the device (masses from the
        Systems).  Returns (positions, velocities, forces, energies), positions, velocities and forces as lists of
        (n_s, 3) arrays, energies (num_systems, 4) at the final positions."""
        def flat(a):
            if isinstance(a, (list, tuple)):
                a = np.concatenate([np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in a])
            return _capi.arr(np.asarray(a, dtype=np.float64).reshape(-1, 3), np.float64).copy()
        pos = flat(positions)
        vel = np.zeros_like(pos) if velocities is None else flat(velocities)
        if pos.shape[0] != self._offsets[-1] or vel.shape != pos.shape:
            raise OpenMMException("positions and velocities must hold every particle of every System of the batch")
        st = _capi.arr(np.broadcast_to(np.asarray(steps, dtype=np.int32), (len(self._systems),)), np.int32)
        mass = _capi.arr([s.getParticleMass(i) for s in self._systems for i in range(s.getNumParticles())],
                         np.float64)
        self._check(self._lib.ix_batch_md_run(self._batch, _capi.ptr(st), float(dt), _capi.ptr(mass), _capi.ptr(pos),
                                              _capi.ptr(vel), _capi.ptr(self._forces), _capi.ptr(self._energies)))
        split = lambda a: [a[self._offsets[s]:self._offsets[s + 1]].copy() for s in range(len(self._systems))]
        return split(pos), split(vel), split(self._forces), self._energies.copy()

    def getCounts(self):
        p, t = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self._lib.ix_batch_get_counts(self._batch, ctypes.byref(p), ctypes.byref(t)))
        return p.value, t.value

    def __del__(self):
        if getattr(self, "_batch", None) and self._batch.value:
            self._lib.ix_batch_destroy(self._batch)
            self._batch = ctypes.c_void_p()
