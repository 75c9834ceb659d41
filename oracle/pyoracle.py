"""ctypes bridge to the FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the
checker.  It evaluates the same System objects the product's Context evaluates, force by force, the way the
reference's Reference platform does (platforms/reference/src/ReferenceInteraxKernels.cpp:71-225).
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None


def build():
    """Compile liboracle.so with the committed Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = _HERE / "liboracle.so"
        if not path.exists():
            build()
        L = ctypes.CDLL(str(path))
        P = ctypes.c_void_p
        L.ox_pair_force.restype = ctypes.c_double
        L.ox_pair_force.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P, P, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_double, P, P]
        L.ox_three_body.restype = ctypes.c_double
        L.ox_three_body.argtypes = [ctypes.c_int, P, P, ctypes.c_int, P, P, P, P, P, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_double, P, P]
        L.ox_slater_overlap.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, P, P]
        L.ox_tang_toennies.argtypes = [ctypes.c_double, P, P]
        L.ox_overlap_taylor_table.argtypes = [P, P]
        L.ox_long_range_coefficients.argtypes = [ctypes.c_int, P, P, P, ctypes.c_double, ctypes.c_int, P, P]
        L.ox_last_abs_energy.restype = ctypes.c_double
        L.ox_last_abs_energy.argtypes = []
        _LIB = L
    return _LIB


class _PairSettings(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("cutoff", ctypes.c_double), ("use_switch", ctypes.c_int),
                ("switch_distance", ctypes.c_double), ("softcore_radius", ctypes.c_double),
                ("num_exclusions", ctypes.c_int), ("exclusions", ctypes.c_void_p)]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def long_range_coefficients(force):
    """The oracle's long-range correction coefficients (coefficient, alchemical coefficient) of a dispersion force."""
    ex = _c(force._exclusion_array(), np.int32)
    s = _PairSettings(force.getNonbondedMethod(), force.getCutoffDistance(), int(force.getUseSwitchingFunction()),
                      force.getSwitchingDistance(), force.getSoftcoreRadius(), len(ex), _ptr(ex))
    params = _c(force._params_array(), np.float64)
    alch = _c(force._alch_array(), np.uint8)
    coef, alch_coef = ctypes.c_double(), ctypes.c_double()
    lib().ox_long_range_coefficients(force.getNumParticles(), ctypes.byref(s), _ptr(params), _ptr(alch),
                                     force.getDampingScale(), int(force.getUseLongRangeCorrection()),
                                     ctypes.byref(coef), ctypes.byref(alch_coef))
    return coef.value, alch_coef.value


def pair_force(term, force, positions, box, lam=1.0, counts=None, overlap_method=None):
    """Energy and forces (N x 3) of one pair force.  term: 0 dispersion, 1 exchange, 2 short range."""
    pos = _c(positions, np.float64)
    n = len(pos)
    boxa = _c(np.asarray(box, dtype=np.float64).reshape(9), np.float64)
    ex = _c(force._exclusion_array(), np.int32)
    s = _PairSettings(force.getNonbondedMethod(), force.getCutoffDistance(), int(force.getUseSwitchingFunction()),
                      force.getSwitchingDistance(), force.getSoftcoreRadius(), len(ex), _ptr(ex))
    params = _c(force._params_array(), np.float64)
    alch = _c(force._alch_array(), np.uint8)
    f = np.zeros((n, 3))
    cnt = ctypes.c_longlong()
    damping = force.getDampingScale() if term == 0 else 1.0
    lrc = int(force.getUseLongRangeCorrection()) if term == 0 else 0
    om = overlap_method if overlap_method is not None else (force.getOverlapMethod() if term != 0 else 0)
    e = lib().ox_pair_force(term, n, _ptr(pos), _ptr(boxa), ctypes.byref(s), _ptr(params), _ptr(alch), damping,
                            lrc, om, lam, _ptr(f), ctypes.byref(cnt))
    if counts is not None:
        counts.append(cnt.value)
    return e, f


def three_body(force, positions, box, lam=1.0, counts=None):
    pos = _c(positions, np.float64)
    n = len(pos)
    boxa = _c(np.asarray(box, dtype=np.float64).reshape(9), np.float64)
    off, part, params, mol, alch = force._site_arrays()
    f = np.zeros((n, 3))
    cnt = ctypes.c_longlong()
    e = lib().ox_three_body(n, _ptr(pos), _ptr(boxa), force.getNumSites(), _ptr(_c(off, np.int32)),
                            _ptr(_c(part, np.int32)), _ptr(_c(params, np.float64)), _ptr(_c(mol, np.int32)),
                            _ptr(_c(alch, np.uint8)), force.getCutoffDistance(), force.getScaleFactor(),
                            force.getDampingMethod(), force.getDampingScale(), force.getCentroidDampingRadius(),
                            int(force.usesPeriodicBoundaryConditions()), lam, _ptr(f), ctypes.byref(cnt))
    if counts is not None:
        counts.append(cnt.value)
    return e, f


def term_of(force):
    from interaxplugin import (InteraxDispersionForce, InteraxExchangeForce, InteraxShortRangeForce,
                               InteraxThreeBodyForce)
    if isinstance(force, InteraxDispersionForce):
        return 0
    if isinstance(force, InteraxExchangeForce):
        return 1
    if isinstance(force, InteraxShortRangeForce):
        return 2
    if isinstance(force, InteraxThreeBodyForce):
        return 3
    return None


def evaluate(system, positions, box=None, parameters=None, groups=0xFFFFFFFF, per_force=False, abs_energy=None):
    """The Reference-platform result for a System: total energy and forces of the forces in `groups`.
    `parameters` maps context parameter names (the alchemical parameters) to values; missing ones default to 1.
    If `abs_energy` is a list, the sum of |pair and triple energies| (before switching; the error scale of the
    reference's tests, tests/TestInteraxPairForce.h:105-142) is appended to it."""
    parameters = parameters or {}
    if box is None:
        box = system.getDefaultPeriodicBoxVectors()
    n = system.getNumParticles()
    energy = 0.0
    forces = np.zeros((n, 3))
    results = []
    total_abs = 0.0
    for force in system._forces:
        term = term_of(force)
        if term is None or not (groups >> force.getForceGroup()) & 1:
            continue
        lam = parameters.get(force.getAlchemicalParameterName(), 1.0)
        if term == 3:
            e, f = three_body(force, positions, box, lam)
        else:
            e, f = pair_force(term, force, positions, box, lam)
        total_abs += lib().ox_last_abs_energy()
        energy += e
        forces += f
        results.append((force, e, f))
    if abs_energy is not None:
        abs_energy.append(total_abs)
    return (energy, forces, results) if per_force else (energy, forces)


def slater_overlap(r, a, b, method=0):
    s = np.zeros(1)
    ds = np.zeros(1)
    lib().ox_slater_overlap(r, a, b, method, _ptr(s), _ptr(ds))
    return s[0], ds[0]


def tang_toennies(x):
    f = np.zeros(3)
    df = np.zeros(3)
    lib().ox_tang_toennies(x, _ptr(f), _ptr(df))
    return f, df


def taylor_table():
    v = np.zeros(63)
    d = np.zeros(63)
    lib().ox_overlap_taylor_table(_ptr(v), _ptr(d))
    return v.reshape(7, 9), d.reshape(7, 9)


class CpuPlatform:
    """The restatement of the reference's CPU platform (oracle/cpu_platform.cpp) for one System: the forces are set up
    once, as the CPU kernels' initialize() does, and evaluate() runs them on `threads` host threads (all cores by
    default): the pair forces in single precision, one pass each with its own neighbor list, the three-body force in
    double precision.  Used as the timed CPU baseline; its results agree with the FP64 oracle to single precision."""

    def __init__(self, system, threads=None):
        L = lib()
        if not getattr(L, "_cpu_ready", False):
            P = ctypes.c_void_p
            L.ox_cpu_threads.restype = ctypes.c_int
            L.ox_cpu_pair_create.restype = P
            L.ox_cpu_pair_create.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_int]
            L.ox_cpu_pair_evaluate.restype = ctypes.c_double
            L.ox_cpu_pair_evaluate.argtypes = [P, P, P, ctypes.c_double, ctypes.c_int, P, P]
            L.ox_cpu_pair_destroy.argtypes = [P]
            L.ox_cpu_three_body_create.restype = P
            L.ox_cpu_three_body_create.argtypes = [ctypes.c_int, P, P, P, P, P, ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int]
            L.ox_cpu_three_body_evaluate.restype = ctypes.c_double
            L.ox_cpu_three_body_evaluate.argtypes = [P, P, P, ctypes.c_double, ctypes.c_int, P, P]
            L.ox_cpu_three_body_destroy.argtypes = [P]
            L._cpu_ready = True
        self._lib = L
        self.threads = int(threads) if threads else L.ox_cpu_threads()
        self._system = system
        self._handles = []
        for force in system._forces:
            term = term_of(force)
            if term is None:
                continue
            if term < 3:
                ex = _c(force._exclusion_array(), np.int32)
                s = _PairSettings(force.getNonbondedMethod(), force.getCutoffDistance(),
                                  int(force.getUseSwitchingFunction()), force.getSwitchingDistance(),
                                  force.getSoftcoreRadius(), len(ex), _ptr(ex))
                params = _c(force._params_array(), np.float64)
                alch = _c(force._alch_array(), np.uint8)
                h = L.ox_cpu_pair_create(term, system.getNumParticles(), ctypes.byref(s), _ptr(params), _ptr(alch),
                                         force.getDampingScale() if term == 0 else 1.0,
                                         int(force.getUseLongRangeCorrection()) if term == 0 else 0,
                                         force.getOverlapMethod() if term != 0 else 0)
            else:
                off, part, params, mol, alch = force._site_arrays()
                h = L.ox_cpu_three_body_create(
                    force.getNumSites(), _ptr(_c(off, np.int32)), _ptr(_c(part, np.int32)),
                    _ptr(_c(params, np.float64)), _ptr(_c(mol, np.int32)), _ptr(_c(alch, np.uint8)),
                    force.getCutoffDistance(), force.getScaleFactor(), force.getDampingMethod(),
                    force.getDampingScale(), force.getCentroidDampingRadius(),
                    int(force.usesPeriodicBoundaryConditions()))
            self._handles.append((force, term, h))

    def evaluate(self, positions, box=None, parameters=None, counts=None):
        """Total energy and forces (N x 3); `counts`, if a list, receives the interacting pairs of the dispersion
        force and the interacting triples."""
        L = self._lib
        parameters = parameters or {}
        if box is None:
            box = self._system.getDefaultPeriodicBoxVectors()
        pos = _c(positions, np.float64)
        boxa = _c(np.asarray(box, dtype=np.float64).reshape(9), np.float64)
        forces = np.zeros((len(pos), 3))
        energy = 0.0
        for force, term, h in self._handles:
            lam = parameters.get(force.getAlchemicalParameterName(), 1.0)
            cnt = ctypes.c_longlong()
            if term < 3:
                energy += L.ox_cpu_pair_evaluate(h, _ptr(pos), _ptr(boxa), lam, self.threads, _ptr(forces),
                                                 ctypes.byref(cnt))
            else:
                energy += L.ox_cpu_three_body_evaluate(h, _ptr(pos), _ptr(boxa), lam, self.threads, _ptr(forces),
                                                       ctypes.byref(cnt))
            if counts is not None and term in (0, 3):
                counts.append(cnt.value)
        return energy, forces

    def __del__(self):
        for _, term, h in getattr(self, "_handles", []):
            if term < 3:
                self._lib.ox_cpu_pair_destroy(h)
            else:
                self._lib.ox_cpu_three_body_destroy(h)
